// lav_build.cu — the LAV layout (include/LAV.h:11-31 of the reference) built
// on the GPU.  The reference ships no LAV builder; this one produces the
// layout its kernel reads (src/scalar/spmv_mtx_lav.cpp:36-79), bit for bit the
// oracle's build_lav:
//   * dense columns: the most populated columns (stable by index) until they
//     hold >= (1-T) of the nonzeros; segment k = dense columns
//     [k*segment_len, (k+1)*segment_len) in that order;
//   * one global row order (rows by dense count, descending, stable), cut into
//     chunks of L rows; inside a chunk each segment orders its rows by their
//     count in that segment (descending, stable) -> out_order;
//   * per (segment, chunk): max-count steps, lane-major, a lane streaming its
//     row's entries of that segment in column order; chunk_offsets_full_mask =
//     first step where not every lane is active; mask[step] = active lanes;
//   * everything else in sparse_part (CRS), in the source order.
// Orders come from stable CUB radix sorts (column density, dense entries by
// segment, rows by dense count, and per segment rows by (chunk, count)), so
// the result does not depend on scheduling; counts use integer atomics.
#include <algorithm>
#include <cstring>
#include <vector>

#include "devsort.cuh"
#include "rvvla_internal.cuh"
#include "scan.cuh"

namespace rvvla {
namespace {

inline unsigned nblk(int64_t n) { return grid_for(n); }

__global__ void lav_col_count_kernel(int64_t nz, const int* __restrict__ Col, int* __restrict__ cnt) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nz) atomicAdd(cnt + Col[k], 1);
}

// descending keys (stable sort ascending on ~key), values = index
__global__ void lav_desc_keys_kernel(int64_t n, const int* __restrict__ cnt, const uint32_t* __restrict__ perm,
                                     uint32_t* __restrict__ key, uint32_t* __restrict__ val) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t idx = perm ? perm[i] : (uint32_t)i;
  key[i] = ~(uint32_t)cnt[idx];
  val[i] = idx;
}

__global__ void lav_to_i64_kernel(int64_t n, const uint32_t* __restrict__ nkey, int64_t* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (int64_t)(~nkey[i]);
}

// dense columns: the prefix of the density order whose running count before
// each column is below the target and whose count is positive
__global__ void lav_ndense_kernel(int64_t n, const int64_t* __restrict__ cum, const uint32_t* __restrict__ nkey,
                                  double target, unsigned long long* __restrict__ ndense) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n && (double)cum[k] < target && ~nkey[k] > 0u) atomicAdd(ndense, 1ull);
}

__global__ void lav_seg_of_kernel(int64_t ndense, int64_t seglen, const uint32_t* __restrict__ corder,
                                  int* __restrict__ seg_of) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < ndense) seg_of[corder[k]] = (int)(k / seglen);
}

// per row: dense and sparse entry counts
__global__ void lav_row_count_kernel(int64_t m, const int* __restrict__ Rst, const int* __restrict__ Col,
                                     const int* __restrict__ seg_of, int64_t* __restrict__ dcount,
                                     int64_t* __restrict__ scount) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  int64_t d = 0, s = 0;
  for (int k = Rst[r]; k < Rst[r + 1]; ++k) {
    if (seg_of[Col[k]] >= 0) ++d;
    else ++s;
  }
  dcount[r] = d;
  scount[r] = s;
}

// per row, in source order: sparse entries into the sparse part; dense
// entries (index, segment, row) into the CRS-ordered dense lists
template <class T>
__global__ void lav_split_kernel(int64_t m, const int* __restrict__ Rst, const int* __restrict__ Col,
                                 const T* __restrict__ Val, const int* __restrict__ seg_of,
                                 const int64_t* __restrict__ drp, const int64_t* __restrict__ srp,
                                 uint32_t* __restrict__ dkey, uint32_t* __restrict__ dval, int* __restrict__ dk,
                                 uint32_t* __restrict__ drow, int* __restrict__ sCol, T* __restrict__ sVal) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  int64_t d = drp[r], s = srp[r];
  for (int k = Rst[r]; k < Rst[r + 1]; ++k) {
    const int sg = seg_of[Col[k]];
    if (sg >= 0) {
      dkey[d] = (uint32_t)sg;
      dval[d] = (uint32_t)d;
      dk[d] = k;
      drow[d] = (uint32_t)r;
      ++d;
    } else {
      sCol[s] = Col[k];
      sVal[s] = Val[k];
      ++s;
    }
  }
}

__global__ void lav_gather_kernel(int64_t nd, const uint32_t* __restrict__ order, const int* __restrict__ dk,
                                  const uint32_t* __restrict__ drow, int* __restrict__ ek,
                                  uint32_t* __restrict__ erow) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nd) return;
  ek[p] = dk[order[p]];
  erow[p] = drow[order[p]];
}

// segbeg[s] = first sorted dense entry of segment s (lower bound)
__global__ void lav_segbeg_kernel(int64_t nseg, int64_t nd, const uint32_t* __restrict__ key,
                                  int64_t* __restrict__ segbeg) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s > nseg) return;
  int64_t lo = 0, hi = nd;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if ((int64_t)key[mid] < s) lo = mid + 1;
    else hi = mid;
  }
  segbeg[s] = lo;
}

__global__ void lav_seg_rows_kernel(int64_t a, int64_t b, const uint32_t* __restrict__ erow,
                                    int64_t* __restrict__ cnt) {
  const int64_t p = a + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < b) atomicAdd((unsigned long long*)(cnt + erow[p]), 1ull);
}

// per segment: rows in global order keyed by (chunk, count descending)
__global__ void lav_chunk_keys_kernel(int64_t m, int64_t L, const uint32_t* __restrict__ gorder,
                                      const int64_t* __restrict__ cnt, uint64_t* __restrict__ key,
                                      uint32_t* __restrict__ val) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= m) return;
  const uint32_t r = gorder[g];
  key[g] = ((uint64_t)(g / L) << 32) | (uint64_t)(~(uint32_t)cnt[r]);
  val[g] = r;
}

// per chunk of one segment: out_order, steps (max count), first partial step
__global__ void lav_chunk_kernel(int64_t m, int64_t L, int64_t cc, int64_t sg, const uint32_t* __restrict__ rows,
                                 const int64_t* __restrict__ cnt, uint32_t* __restrict__ oo,
                                 int64_t* __restrict__ steps, int* __restrict__ minc) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cc) return;
  const int64_t r0 = c * L, nrows = min(m, r0 + L) - r0;
  uint32_t* o = oo + (c + cc * sg) * L;
  for (int64_t i = 0; i < L; ++i) o[i] = i < nrows ? rows[r0 + i] : (uint32_t)(m > 0 ? m - 1 : 0);
  steps[c] = nrows > 0 ? cnt[rows[r0]] : 0;
  minc[c] = nrows < L ? 0 : (int)cnt[rows[r0 + L - 1]];
}

__global__ void lav_offsets_kernel(int64_t cc, int64_t sg, const int64_t* __restrict__ sx,
                                   const int* __restrict__ minc, int* __restrict__ co, int* __restrict__ cf,
                                   uint64_t* __restrict__ seg_steps) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c > cc) return;
  co[(cc + 1) * sg + c] = (int)sx[c];
  if (c < cc) cf[sg * cc + c] = (int)sx[c] + minc[c];
  else seg_steps[sg] = (uint64_t)sx[cc];
}

__global__ void lav_segptr_kernel(int64_t nseg, const uint64_t* __restrict__ seg_steps, uint64_t* __restrict__ sp) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    uint64_t a = 0;
    sp[0] = 0;
    for (int64_t s = 0; s < nseg; ++s) {
      a += seg_steps[s];
      sp[s + 1] = a;
    }
  }
}

// lane i of chunk c streams its row's entries of the segment; mask[step] is
// the number of lanes still active (lanes are ordered by count, descending)
template <class T>
__global__ void lav_fill_kernel(int64_t m, int64_t L, int64_t cc, int64_t sg, const uint64_t* __restrict__ sp,
                                const int* __restrict__ co, const uint32_t* __restrict__ oo,
                                const int64_t* __restrict__ cnt, const int64_t* __restrict__ srp,
                                const int* __restrict__ ek, const int* __restrict__ Col, const T* __restrict__ Val,
                                uint32_t* __restrict__ col, T* __restrict__ val, uint16_t* __restrict__ mk) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cc * L) return;
  const int64_t c = t / L, i = t % L;
  const int64_t nrows = min(m, (c + 1) * L) - c * L;
  if (i >= nrows) return;
  const int64_t base = (int64_t)sp[sg] + co[(cc + 1) * sg + c];
  const uint32_t r = oo[(c + cc * sg) * L + i];
  const int64_t e0 = srp[r], n_i = cnt[r];
  const int64_t n_next = (i + 1 < nrows) ? cnt[oo[(c + cc * sg) * L + i + 1]] : 0;
  for (int64_t q = 0; q < n_i; ++q) {
    const int64_t dst = (base + q) * L + i;
    const int k = ek[e0 + q];
    col[dst] = (uint32_t)Col[k];
    val[dst] = Val[k];
  }
  for (int64_t q = n_next; q < n_i; ++q) mk[base + q] = (uint16_t)(i + 1);
}

__global__ void lav_slot_kernel(int64_t m, int64_t L, const uint32_t* __restrict__ gorder, uint8_t* __restrict__ slot) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < m) slot[gorder[g]] = (uint8_t)(g % L);
}

__global__ void lav_lane_of_slot_kernel(int64_t m, int64_t L, int64_t cc, int64_t nseg,
                                        const uint32_t* __restrict__ oo, const uint8_t* __restrict__ slot,
                                        uint8_t* __restrict__ lo) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nseg * cc * L) return;
  const int64_t q = t / L, i = t % L, c = q % cc;
  const int64_t nrows = min(m, (c + 1) * L) - c * L;
  if (i < nrows) lo[q * L + slot[oo[q * L + i]]] = (uint8_t)i;
  else lo[q * L + i] = (uint8_t)i;
}

__global__ void lav_long_chunks_kernel(int64_t cc, int64_t nseg, const int* __restrict__ co, int64_t long_steps,
                                       unsigned long long* __restrict__ lc) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cc) return;
  int64_t steps = 0;
  for (int64_t s = 0; s < nseg; ++s) steps += co[(cc + 1) * s + c + 1] - co[(cc + 1) * s + c];
  if (steps >= long_steps) atomicMax(lc, (unsigned long long)(c + 1));
}

__global__ void lav_i64_to_i32_kernel(int64_t n, const int64_t* __restrict__ in, int* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (int)in[i];
}

template <class T>
int dev_alloc(T** p, int64_t n) {
  RVVLA_CUDA(cudaMalloc(p, (size_t)std::max<int64_t>(n, 1) * sizeof(T)));
  return RVVLA_OK;
}

}  // namespace

template <class T>
int lav_build_gpu(const rvvla_crs* src, int64_t L, double Tthr, int64_t seglen, int64_t long_steps,
                  rvvla_lav_owned* out, cudaStream_t st) {
  const int64_t m = src->m, n = src->n, nz = src->nz;
  const T* Val = static_cast<const T*>(src->Val);
  rvvla_lav& h = out->h;
  h.SIMD_Lanes = L; h.m = m; h.n = n; h.nz = nz; h.segment_len = seglen; h.T = Tthr;
  const int64_t cc = (m + L - 1) / L;
  h.chunk_count = cc;
  int rc = 0;
  // ---- dense columns
  Scratch s_ccnt, s_k1, s_v1, s_k2, s_corder, s_cum, s_cnt64, s_nd;
  RVVLA_CUDA(s_ccnt.alloc((size_t)std::max<int64_t>(n, 1) * 4, st));
  RVVLA_CUDA(cudaMemsetAsync(s_ccnt.p, 0, (size_t)std::max<int64_t>(n, 1) * 4, st));
  if (nz > 0) lav_col_count_kernel<<<nblk(nz), 256, 0, st>>>(nz, src->Col, s_ccnt.as<int>());
  RVVLA_CUDA(s_k1.alloc((size_t)std::max<int64_t>(n, 1) * 4, st));
  RVVLA_CUDA(s_v1.alloc((size_t)std::max<int64_t>(n, 1) * 4, st));
  RVVLA_CUDA(s_k2.alloc((size_t)std::max<int64_t>(n, 1) * 4, st));
  RVVLA_CUDA(s_corder.alloc((size_t)std::max<int64_t>(n, 1) * 4, st));
  if (n > 0) {
    lav_desc_keys_kernel<<<nblk(n), 256, 0, st>>>(n, s_ccnt.as<int>(), nullptr, s_k1.as<uint32_t>(),
                                                   s_v1.as<uint32_t>());
    if ((rc = radix_sort_pairs(s_k1.as<uint32_t>(), s_k2.as<uint32_t>(), s_v1.as<uint32_t>(),
                               s_corder.as<uint32_t>(), n, 32, st)))
      return rc;
  }
  RVVLA_CUDA(s_cnt64.alloc((size_t)(n + 1) * 8, st));
  RVVLA_CUDA(s_cum.alloc((size_t)(n + 1) * 8, st));
  RVVLA_CUDA(s_nd.alloc(8, st));
  RVVLA_CUDA(cudaMemsetAsync(s_nd.p, 0, 8, st));
  if (n > 0) {
    lav_to_i64_kernel<<<nblk(n), 256, 0, st>>>(n, s_k2.as<uint32_t>(), s_cnt64.as<int64_t>());
    if ((rc = exclusive_scan_i64(s_cnt64.as<int64_t>(), s_cum.as<int64_t>(), n, st))) return rc;
    lav_ndense_kernel<<<nblk(n), 256, 0, st>>>(n, s_cum.as<int64_t>(), s_k2.as<uint32_t>(), (1.0 - Tthr) * (double)nz,
                                                s_nd.as<unsigned long long>());
  }
  RVVLA_LAUNCHED("lav dense-column kernels");
  unsigned long long ndense_u = 0;
  RVVLA_CUDA(cudaMemcpyAsync(&ndense_u, s_nd.p, 8, cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaStreamSynchronize(st));
  const int64_t ndense = (int64_t)ndense_u;
  const int64_t nseg = (ndense + seglen - 1) / seglen;
  h.segment_count = nseg;
  Scratch s_seg;
  RVVLA_CUDA(s_seg.alloc((size_t)std::max<int64_t>(n, 1) * 4, st));
  RVVLA_CUDA(cudaMemsetAsync(s_seg.p, 0xFF, (size_t)std::max<int64_t>(n, 1) * 4, st));
  if (ndense > 0)
    lav_seg_of_kernel<<<nblk(ndense), 256, 0, st>>>(ndense, seglen, s_corder.as<uint32_t>(), s_seg.as<int>());
  // ---- split the entries: sparse part (source order) and dense entries
  Scratch s_dcnt, s_scnt, s_drp, s_srp;
  RVVLA_CUDA(s_dcnt.alloc((size_t)(m + 1) * 8, st));
  RVVLA_CUDA(s_scnt.alloc((size_t)(m + 1) * 8, st));
  RVVLA_CUDA(s_drp.alloc((size_t)(m + 1) * 8, st));
  RVVLA_CUDA(s_srp.alloc((size_t)(m + 1) * 8, st));
  if (m > 0) {
    lav_row_count_kernel<<<nblk(m), 256, 0, st>>>(m, src->Rst, src->Col, s_seg.as<int>(), s_dcnt.as<int64_t>(),
                                                   s_scnt.as<int64_t>());
    if ((rc = exclusive_scan_i64(s_dcnt.as<int64_t>(), s_drp.as<int64_t>(), m, st))) return rc;
    if ((rc = exclusive_scan_i64(s_scnt.as<int64_t>(), s_srp.as<int64_t>(), m, st))) return rc;
  } else {
    RVVLA_CUDA(cudaMemsetAsync(s_drp.p, 0, 8, st));
    RVVLA_CUDA(cudaMemsetAsync(s_srp.p, 0, 8, st));
  }
  int64_t tot[2] = {0, 0};
  RVVLA_CUDA(cudaMemcpyAsync(&tot[0], s_drp.as<int64_t>() + m, 8, cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaMemcpyAsync(&tot[1], s_srp.as<int64_t>() + m, 8, cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaStreamSynchronize(st));
  const int64_t nd = tot[0], nsp = tot[1];
  if ((rc = dev_alloc(&out->sp_Rst, m + 1))) return rc;
  if ((rc = dev_alloc(&out->sp_Col, nsp))) return rc;
  if ((rc = dev_alloc(reinterpret_cast<T**>(&out->sp_Val), nsp))) return rc;
  Scratch s_dkey, s_dval, s_dk, s_drow, s_skey, s_order, s_ek, s_erow;
  RVVLA_CUDA(s_dkey.alloc((size_t)std::max<int64_t>(nd, 1) * 4, st));
  RVVLA_CUDA(s_dval.alloc((size_t)std::max<int64_t>(nd, 1) * 4, st));
  RVVLA_CUDA(s_dk.alloc((size_t)std::max<int64_t>(nd, 1) * 4, st));
  RVVLA_CUDA(s_drow.alloc((size_t)std::max<int64_t>(nd, 1) * 4, st));
  if (m > 0) {
    lav_split_kernel<T><<<nblk(m), 256, 0, st>>>(m, src->Rst, src->Col, Val, s_seg.as<int>(), s_drp.as<int64_t>(),
                                                  s_srp.as<int64_t>(), s_dkey.as<uint32_t>(), s_dval.as<uint32_t>(),
                                                  s_dk.as<int>(), s_drow.as<uint32_t>(), out->sp_Col,
                                                  static_cast<T*>(out->sp_Val));
    lav_i64_to_i32_kernel<<<nblk(m + 1), 256, 0, st>>>(m + 1, s_srp.as<int64_t>(), out->sp_Rst);
  } else {
    RVVLA_CUDA(cudaMemsetAsync(out->sp_Rst, 0, 4, st));
  }
  RVVLA_LAUNCHED("lav split kernels");
  // dense entries grouped by segment, source order inside a segment
  RVVLA_CUDA(s_skey.alloc((size_t)std::max<int64_t>(nd, 1) * 4, st));
  RVVLA_CUDA(s_order.alloc((size_t)std::max<int64_t>(nd, 1) * 4, st));
  RVVLA_CUDA(s_ek.alloc((size_t)std::max<int64_t>(nd, 1) * 4, st));
  RVVLA_CUDA(s_erow.alloc((size_t)std::max<int64_t>(nd, 1) * 4, st));
  if (nd > 0) {
    if ((rc = radix_sort_pairs(s_dkey.as<uint32_t>(), s_skey.as<uint32_t>(), s_dval.as<uint32_t>(),
                               s_order.as<uint32_t>(), nd, bits_for((uint64_t)std::max<int64_t>(nseg, 1)), st)))
      return rc;
    lav_gather_kernel<<<nblk(nd), 256, 0, st>>>(nd, s_order.as<uint32_t>(), s_dk.as<int>(), s_drow.as<uint32_t>(),
                                                 s_ek.as<int>(), s_erow.as<uint32_t>());
  }
  Scratch s_segbeg;
  RVVLA_CUDA(s_segbeg.alloc((size_t)(nseg + 1) * 8, st));
  lav_segbeg_kernel<<<nblk(nseg + 1), 256, 0, st>>>(nseg, nd, s_skey.as<uint32_t>(), s_segbeg.as<int64_t>());
  // rows by dense count, descending, stable
  if ((rc = dev_alloc(&out->row_order, m))) return rc;
  {
    Scratch s_rk, s_rv, s_rk2, s_dc32;
    RVVLA_CUDA(s_rk.alloc((size_t)std::max<int64_t>(m, 1) * 4, st));
    RVVLA_CUDA(s_rv.alloc((size_t)std::max<int64_t>(m, 1) * 4, st));
    RVVLA_CUDA(s_rk2.alloc((size_t)std::max<int64_t>(m, 1) * 4, st));
    RVVLA_CUDA(s_dc32.alloc((size_t)std::max<int64_t>(m, 1) * 4, st));
    if (m > 0) {
      lav_i64_to_i32_kernel<<<nblk(m), 256, 0, st>>>(m, s_dcnt.as<int64_t>(), s_dc32.as<int>());
      lav_desc_keys_kernel<<<nblk(m), 256, 0, st>>>(m, s_dc32.as<int>(), nullptr, s_rk.as<uint32_t>(),
                                                     s_rv.as<uint32_t>());
      if ((rc = radix_sort_pairs(s_rk.as<uint32_t>(), s_rk2.as<uint32_t>(), s_rv.as<uint32_t>(), out->row_order, m,
                                 32, st)))
        return rc;
    }
  }
  std::vector<int64_t> segbeg((size_t)nseg + 1, 0);
  RVVLA_CUDA(cudaMemcpyAsync(segbeg.data(), s_segbeg.p, (size_t)(nseg + 1) * 8, cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaStreamSynchronize(st));
  // ---- pass 1: per segment, chunk order and steps
  if ((rc = dev_alloc(&out->chunk_offsets, (cc + 1) * nseg))) return rc;
  if ((rc = dev_alloc(&out->chunk_offsets_full_mask, cc * nseg))) return rc;
  if ((rc = dev_alloc(&out->segment_ptr, nseg + 1))) return rc;
  if ((rc = dev_alloc(&out->out_order, nseg * cc * L))) return rc;
  Scratch s_rc, s_rsrp, s_ck, s_ck2, s_cv, s_rows, s_steps, s_sx, s_minc, s_segsteps;
  RVVLA_CUDA(s_rc.alloc((size_t)(m + 1) * 8, st));
  RVVLA_CUDA(s_rsrp.alloc((size_t)(m + 1) * 8, st));
  RVVLA_CUDA(s_ck.alloc((size_t)std::max<int64_t>(m, 1) * 8, st));
  RVVLA_CUDA(s_ck2.alloc((size_t)std::max<int64_t>(m, 1) * 8, st));
  RVVLA_CUDA(s_cv.alloc((size_t)std::max<int64_t>(m, 1) * 4, st));
  RVVLA_CUDA(s_rows.alloc((size_t)std::max<int64_t>(m, 1) * 4, st));
  RVVLA_CUDA(s_steps.alloc((size_t)(cc + 1) * 8, st));
  RVVLA_CUDA(s_sx.alloc((size_t)(cc + 1) * 8, st));
  RVVLA_CUDA(s_minc.alloc((size_t)std::max<int64_t>(cc, 1) * 4, st));
  RVVLA_CUDA(s_segsteps.alloc((size_t)std::max<int64_t>(nseg, 1) * 8, st));
  const int key_bits = 32 + bits_for((uint64_t)std::max<int64_t>(cc, 1));
  // per segment: every row's entry count in it and the first entry of each row
  auto seg_rows = [&](int64_t sg) -> int {
    RVVLA_CUDA(cudaMemsetAsync(s_rc.p, 0, (size_t)(m + 1) * 8, st));
    const int64_t a = segbeg[(size_t)sg], b = segbeg[(size_t)sg + 1];
    if (b > a)
      lav_seg_rows_kernel<<<nblk(b - a), 256, 0, st>>>(a, b, s_erow.as<uint32_t>(), s_rc.as<int64_t>());
    RVVLA_LAUNCHED("lav_seg_rows_kernel");
    return RVVLA_OK;
  };
  for (int64_t sg = 0; sg < nseg; ++sg) {
    if ((rc = seg_rows(sg))) return rc;
    lav_chunk_keys_kernel<<<nblk(m), 256, 0, st>>>(m, L, out->row_order, s_rc.as<int64_t>(), s_ck.as<uint64_t>(),
                                                    s_cv.as<uint32_t>());
    if ((rc = radix_sort_pairs(s_ck.as<uint64_t>(), s_ck2.as<uint64_t>(), s_cv.as<uint32_t>(), s_rows.as<uint32_t>(),
                               m, key_bits, st)))
      return rc;
    lav_chunk_kernel<<<nblk(cc), 256, 0, st>>>(m, L, cc, sg, s_rows.as<uint32_t>(), s_rc.as<int64_t>(),
                                               out->out_order, s_steps.as<int64_t>(), s_minc.as<int>());
    if ((rc = exclusive_scan_i64(s_steps.as<int64_t>(), s_sx.as<int64_t>(), cc, st))) return rc;
    lav_offsets_kernel<<<nblk(cc + 1), 256, 0, st>>>(cc, sg, s_sx.as<int64_t>(), s_minc.as<int>(),
                                                      out->chunk_offsets, out->chunk_offsets_full_mask,
                                                      s_segsteps.as<uint64_t>());
    RVVLA_LAUNCHED("lav chunk kernels");
  }
  lav_segptr_kernel<<<1, 32, 0, st>>>(nseg, s_segsteps.as<uint64_t>(), out->segment_ptr);
  RVVLA_LAUNCHED("lav_segptr_kernel");
  uint64_t nsteps = 0;
  RVVLA_CUDA(cudaMemcpyAsync(&nsteps, out->segment_ptr + nseg, 8, cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaStreamSynchronize(st));
  h.n_steps = (int64_t)nsteps;
  // ---- pass 2: lane-major steps
  if ((rc = dev_alloc(&out->mask, (int64_t)nsteps))) return rc;
  if ((rc = dev_alloc(&out->col_id, (int64_t)nsteps * L))) return rc;
  if ((rc = dev_alloc(reinterpret_cast<T**>(&out->val), (int64_t)nsteps * L))) return rc;
  RVVLA_CUDA(cudaMemsetAsync(out->mask, 0, std::max<size_t>(nsteps, 1) * 2, st));
  RVVLA_CUDA(cudaMemsetAsync(out->col_id, 0, std::max<size_t>(nsteps * L, 1) * 4, st));
  RVVLA_CUDA(cudaMemsetAsync(out->val, 0, std::max<size_t>(nsteps * L, 1) * sizeof(T), st));
  for (int64_t sg = 0; sg < nseg; ++sg) {
    if ((rc = seg_rows(sg))) return rc;
    if ((rc = exclusive_scan_i64(s_rc.as<int64_t>(), s_rsrp.as<int64_t>(), m, st))) return rc;
    // row starts inside this segment's slice of the sorted dense entries
    lav_fill_kernel<T><<<nblk(cc * L), 256, 0, st>>>(m, L, cc, sg, out->segment_ptr, out->chunk_offsets,
                                                      out->out_order, s_rc.as<int64_t>(), s_rsrp.as<int64_t>(),
                                                      s_ek.as<int>() + segbeg[(size_t)sg], src->Col, Val,
                                                      out->col_id, static_cast<T*>(out->val), out->mask);
    RVVLA_LAUNCHED("lav_fill_kernel");
  }
  // ---- derived data of the one-pass kernel
  if (L <= 256) {
    if ((rc = dev_alloc(&out->lane_of_slot, nseg * cc * L))) return rc;
    Scratch s_slot;
    RVVLA_CUDA(s_slot.alloc((size_t)std::max<int64_t>(m, 1), st));
    if (m > 0) lav_slot_kernel<<<nblk(m), 256, 0, st>>>(m, L, out->row_order, s_slot.as<uint8_t>());
    if (nseg * cc * L > 0)
      lav_lane_of_slot_kernel<<<nblk(nseg * cc * L), 256, 0, st>>>(m, L, cc, nseg, out->out_order,
                                                                  s_slot.as<uint8_t>(), out->lane_of_slot);
    RVVLA_LAUNCHED("lav lane_of_slot kernels");
  }
  {
    Scratch s_lc;
    RVVLA_CUDA(s_lc.alloc(8, st));
    RVVLA_CUDA(cudaMemsetAsync(s_lc.p, 0, 8, st));
    if (cc > 0 && nseg > 0)
      lav_long_chunks_kernel<<<nblk(cc), 256, 0, st>>>(cc, nseg, out->chunk_offsets, long_steps,
                                                        s_lc.as<unsigned long long>());
    RVVLA_LAUNCHED("lav_long_chunks_kernel");
    unsigned long long lc = 0;
    RVVLA_CUDA(cudaMemcpyAsync(&lc, s_lc.p, 8, cudaMemcpyDeviceToHost, st));
    RVVLA_CUDA(cudaStreamSynchronize(st));
    h.long_chunks = (int64_t)lc;
  }
  h.chunk_offsets = out->chunk_offsets;
  h.chunk_offsets_full_mask = out->chunk_offsets_full_mask;
  h.segment_ptr = out->segment_ptr;
  h.out_order = out->out_order;
  h.mask = out->mask;
  h.val = out->val;
  h.col_id = out->col_id;
  h.row_order = out->row_order;
  h.lane_of_slot = out->lane_of_slot;
  h.sparse_part.m = m;
  h.sparse_part.n = n;
  h.sparse_part.nz = nsp;
  h.sparse_part.Rst = out->sp_Rst;
  h.sparse_part.Col = out->sp_Col;
  h.sparse_part.Val = out->sp_Val;
  h.sparse_part.plan = nullptr;
  h.sparse_part.plan_tiles = 0;
  h.sparse_part.plan_kind = 0;
  RVVLA_CUDA(cudaStreamSynchronize(st));
  return RVVLA_OK;
}

template int lav_build_gpu<double>(const rvvla_crs*, int64_t, double, int64_t, int64_t, rvvla_lav_owned*,
                                   cudaStream_t);
template int lav_build_gpu<float>(const rvvla_crs*, int64_t, double, int64_t, int64_t, rvvla_lav_owned*,
                                  cudaStream_t);

}  // namespace rvvla
