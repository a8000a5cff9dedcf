// lav_build.h — host builder of the LAV layout (include/LAV.h:11-31 of the
// reference), shared by the CUDA entry point.  The reference ships no LAV
// builder; this one follows the layout its kernel reads
// (src/scalar/spmv_mtx_lav.cpp:36-79):
//   * dense columns: the most populated columns (stable by index) until they
//     hold >= (1-T) of the nonzeros; segment k = dense columns
//     [k*segment_len, (k+1)*segment_len) in that order;
//   * one global row order (rows by dense count, descending, stable), cut into
//     chunks of L rows; inside a chunk each segment orders its rows by their
//     count in that segment (descending, stable) -> out_order;
//   * per (segment, chunk): max-count steps, lane-major, a lane streaming its
//     row's entries of that segment in column order; chunk_offsets_full_mask =
//     first step where not every lane is active (incomplete chunks: none);
//     mask[step] = active lanes (a prefix of the chunk);
//   * everything else in sparse_part (CRS).
// Cost O(nnz + segment_count*m): a stable counting sort of the dense entries
// by segment, then per segment a row histogram (OpenMP over segments).
#pragma once
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <vector>

namespace rvvla {

template <class T>
struct LavHost {
  int64_t L = 8, m = 0, n = 0, nz = 0, nseg = 0, cc = 0, seglen = 0;
  double thr = 0.2;
  std::vector<int> co, cf, sRst, sCol;
  std::vector<uint64_t> sp;
  std::vector<uint32_t> oo, col;
  std::vector<uint16_t> mk;
  std::vector<T> val, sVal;
  // derived for the one-pass GPU kernel (not part of the reference layout):
  // the global row order, and per (segment, chunk, slot j) the lane that
  // holds row_order[chunk*L + j] in that segment (only for L <= 256)
  std::vector<uint32_t> row_order;
  std::vector<uint8_t> lane_of_slot;
};

template <class T>
void lav_build_host(const int* Rst, const int* Col, const T* Val, int64_t m, int64_t n, int64_t nz, int64_t L,
                    double Tthr, int64_t seglen, LavHost<T>& o) {
  o.L = L; o.m = m; o.n = n; o.nz = nz; o.thr = Tthr; o.seglen = seglen;
  std::vector<int64_t> ccount((size_t)n, 0);
  for (int64_t k = 0; k < nz; ++k) ccount[(size_t)Col[k]]++;
  std::vector<int> corder((size_t)n);
  std::iota(corder.begin(), corder.end(), 0);
  std::stable_sort(corder.begin(), corder.end(), [&](int a, int b) { return ccount[(size_t)a] > ccount[(size_t)b]; });
  const double target = (1.0 - Tthr) * (double)nz;
  int64_t ndense = 0, cum = 0;
  while (ndense < n && (double)cum < target && ccount[(size_t)corder[(size_t)ndense]] > 0) {
    cum += ccount[(size_t)corder[(size_t)ndense]];
    ndense++;
  }
  std::vector<int> seg_of((size_t)n, -1);
  for (int64_t k = 0; k < ndense; ++k) seg_of[(size_t)corder[(size_t)k]] = (int)(k / seglen);
  const int64_t nseg = (ndense + seglen - 1) / seglen;
  const int64_t cc = (m + L - 1) / L;
  o.nseg = nseg;
  o.cc = cc;
  std::vector<int64_t> dcount((size_t)m, 0);
  o.sRst.assign((size_t)m + 1, 0);
  std::vector<int64_t> segbeg((size_t)nseg + 1, 0);
  for (int64_t r = 0; r < m; ++r)
    for (int64_t k = Rst[r]; k < Rst[r + 1]; ++k) {
      const int sg = seg_of[(size_t)Col[k]];
      if (sg >= 0) { dcount[(size_t)r]++; segbeg[(size_t)sg + 1]++; }
      else o.sRst[(size_t)r + 1]++;
    }
  for (int64_t r = 0; r < m; ++r) o.sRst[(size_t)r + 1] += o.sRst[(size_t)r];
  for (int64_t sg = 0; sg < nseg; ++sg) segbeg[(size_t)sg + 1] += segbeg[(size_t)sg];
  // dense entries grouped by segment; inside a segment row-major with
  // ascending columns (a stable counting sort of the CRS order)
  std::vector<uint32_t> erow((size_t)segbeg[(size_t)nseg]);
  std::vector<int64_t> ek((size_t)segbeg[(size_t)nseg]);
  {
    std::vector<int64_t> cur(segbeg.begin(), segbeg.end() - 1);
    for (int64_t r = 0; r < m; ++r)
      for (int64_t k = Rst[r]; k < Rst[r + 1]; ++k) {
        const int sg = seg_of[(size_t)Col[k]];
        if (sg >= 0) {
          const int64_t q = cur[(size_t)sg]++;
          erow[(size_t)q] = (uint32_t)r;
          ek[(size_t)q] = k;
        } else {
          o.sCol.push_back(Col[k]);
          o.sVal.push_back(Val[k]);
        }
      }
  }
  std::vector<uint32_t> gorder((size_t)m);
  std::iota(gorder.begin(), gorder.end(), 0u);
  std::stable_sort(gorder.begin(), gorder.end(), [&](uint32_t a, uint32_t b) { return dcount[a] > dcount[b]; });
  o.row_order = gorder;
  o.co.assign((size_t)((cc + 1) * nseg), 0);
  o.cf.assign((size_t)(cc * nseg), 0);
  o.sp.assign((size_t)nseg + 1, 0);
  o.oo.assign((size_t)(nseg * cc * L), (uint32_t)(m > 0 ? m - 1 : 0));
  // per segment: every row's count and first entry in that segment
  auto seg_rows = [&](int64_t sg, std::vector<int32_t>& scount, std::vector<int64_t>& srp) {
    std::fill(scount.begin(), scount.end(), 0);
    for (int64_t q = segbeg[(size_t)sg]; q < segbeg[(size_t)sg + 1]; ++q) scount[erow[(size_t)q]]++;
    srp[0] = segbeg[(size_t)sg];
    for (int64_t r = 0; r < m; ++r) srp[(size_t)r + 1] = srp[(size_t)r] + scount[(size_t)r];
  };
  auto chunk_rows = [&](int64_t c, const std::vector<int32_t>& scount, std::vector<uint32_t>& rows) {
    const int64_t r0 = c * L, r1 = std::min(m, r0 + L);
    rows.assign(gorder.begin() + r0, gorder.begin() + r1);
    std::stable_sort(rows.begin(), rows.end(), [&](uint32_t a, uint32_t b) { return scount[a] > scount[b]; });
  };
  // pass 1: steps per segment (chunk_offsets are segment-relative)
#pragma omp parallel
  {
    std::vector<int32_t> scount((size_t)m);
    std::vector<int64_t> srp((size_t)m + 1);
    std::vector<uint32_t> rows;
#pragma omp for schedule(dynamic, 1)
    for (int64_t sg = 0; sg < nseg; ++sg) {
      seg_rows(sg, scount, srp);
      int64_t step = 0;
      for (int64_t c = 0; c < cc; ++c) {
        chunk_rows(c, scount, rows);
        const int64_t maxc = rows.empty() ? 0 : scount[rows[0]];
        const int64_t minc = ((int64_t)rows.size() < L) ? 0 : scount[rows.back()];
        for (size_t i = 0; i < rows.size(); ++i) o.oo[(size_t)((c + cc * sg) * L) + i] = rows[i];
        o.co[(size_t)((cc + 1) * sg + c)] = (int)step;
        o.cf[(size_t)(sg * cc + c)] = (int)(step + minc);
        step += maxc;
      }
      o.co[(size_t)((cc + 1) * sg + cc)] = (int)step;
      o.sp[(size_t)sg + 1] = (uint64_t)step;
    }
  }
  for (int64_t sg = 0; sg < nseg; ++sg) o.sp[(size_t)sg + 1] += o.sp[(size_t)sg];
  const int64_t nsteps = (int64_t)o.sp[(size_t)nseg];
  o.mk.assign((size_t)nsteps, 0);
  o.col.assign((size_t)(nsteps * L), 0u);
  o.val.assign((size_t)(nsteps * L), T(0));
  // pass 2: lane-major steps; lane i of a chunk streams its row's entries
#pragma omp parallel
  {
    std::vector<int32_t> scount((size_t)m);
    std::vector<int64_t> srp((size_t)m + 1);
#pragma omp for schedule(dynamic, 1)
    for (int64_t sg = 0; sg < nseg; ++sg) {
      seg_rows(sg, scount, srp);
      const int64_t base = (int64_t)o.sp[(size_t)sg];
      for (int64_t c = 0; c < cc; ++c) {
        const int64_t st = o.co[(size_t)((cc + 1) * sg + c)];
        const int64_t nrows = std::min(m, (c + 1) * L) - c * L;
        for (int64_t i = 0; i < nrows; ++i) {
          const uint32_t r = o.oo[(size_t)((c + cc * sg) * L + i)];
          const int64_t e0 = srp[r], cnt = scount[r];
          for (int64_t q = 0; q < cnt; ++q) {
            const size_t dst = (size_t)((base + st + q) * L + i);
            const int64_t k = ek[(size_t)(e0 + q)];
            o.col[dst] = (uint32_t)Col[k];
            o.val[dst] = Val[k];
            o.mk[(size_t)(base + st + q)]++;
          }
        }
      }
    }
  }
  // slot -> lane map (identity for the padding slots of the last chunk)
  if (L <= 256) {
    std::vector<uint8_t> slot_of((size_t)m);
    for (int64_t g = 0; g < m; ++g) slot_of[o.row_order[(size_t)g]] = (uint8_t)(g % L);
    o.lane_of_slot.assign((size_t)(nseg * cc * L), 0);
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < nseg * cc; ++q) {
      const int64_t c = q % cc;
      const int64_t nrows = std::min(m, (c + 1) * L) - c * L;
      uint8_t* lo = &o.lane_of_slot[(size_t)(q * L)];
      for (int64_t i = 0; i < L; ++i) lo[i] = (uint8_t)i;
      for (int64_t i = 0; i < nrows; ++i) lo[slot_of[o.oo[(size_t)(q * L + i)]]] = (uint8_t)i;
    }
  }
}

}  // namespace rvvla
