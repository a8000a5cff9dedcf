// vnec_build.cpp — host builder of spMtxVNEC structures (include/VNEC.h of
// the reference builds them on the host, in its constructor; the S and D
// auxiliary arrays are defined there only by use, in
// src/rvv/spmv_mtx_vnec.cpp).
//
//   partition : merge path of (row ends, nonzero indices) into
//               NUM_THREADS_VNEC pieces (VNEC.h:89-100, MergePathDivide
//               spmv_mtx_vnec.cpp:42-71);
//   compaction: per piece, its distinct columns ascending (use_x_indices) and
//               each nonzero's rank among them (ecr_indices) (VNEC.h:104-140);
//   groups    : per row, windows of nLanes consecutive compacted columns
//               (col_start, v_row_ptr) with values in val_align
//               (VNEC.h:147-177; the reference computes them only to count);
//   IRD       : nnz / (groups * nLanes); variant L if m >= 2,000,000, else D
//               if IRD >= 0.437 (fp32) / 0.477 (fp64), else S (VNEC.h:218-226,
//               SpB_mxv_VNEC.h:22-25);
//   S         : whole rows per piece (rows of the merge-path row ranges);
//               rows shorter than nLanes in cross-row groups of nLanes rows
//               (by length, descending, stable; padded with value 0 /
//               compacted column 0), the rest in-row; every row in one task.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "vnec_build.h"

namespace rvvla {

static void merge_path_host(int64_t diagonal, const int* a, int64_t a_len, int64_t b_len, int* x, int* y) {
  int64_t lo = std::max<int64_t>(diagonal - b_len, 0), hi = std::min<int64_t>(diagonal, a_len);
  while (lo < hi) {
    const int64_t piv = (lo + hi) >> 1;
    if ((int64_t)a[piv] <= diagonal - piv - 1) lo = piv + 1;
    else hi = piv;
  }
  *x = (int)std::min(lo, a_len);
  *y = (int)(diagonal - lo);
}

template <class T>
void vnec_build_host(const int* Rst, const int* Col, const T* Val, int64_t m, int64_t n, int64_t nnz, int64_t NT,
                     int force, int nL, double thr, VnecHost<T>& o) {
  o = VnecHost<T>();
  o.NT = (int)NT;
  o.nL = nL;
  const int64_t items = nnz + m;
  const int64_t ipt = (items + NT - 1) / NT;
  o.tcs.assign((size_t)(2 * NT), 0);
  o.tce.assign((size_t)(2 * NT), 0);
  for (int64_t t = 0; t < NT; ++t) {
    const int64_t d0 = std::min(ipt * t, items), d1 = std::min(d0 + ipt, items);
    merge_path_host(d0, Rst + 1, m, nnz, &o.tcs[(size_t)(2 * t)], &o.tcs[(size_t)(2 * t + 1)]);
    merge_path_host(d1, Rst + 1, m, nnz, &o.tce[(size_t)(2 * t)], &o.tce[(size_t)(2 * t + 1)]);
  }
  // compaction per piece
  o.ecr.assign((size_t)nnz, 0);
  o.nec.assign((size_t)NT, 0);
  std::vector<std::vector<int>> used((size_t)NT);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t t = 0; t < NT; ++t) {
    const int y0 = o.tcs[(size_t)(2 * t + 1)], y1 = o.tce[(size_t)(2 * t + 1)];
    std::vector<int>& u = used[(size_t)t];
    u.assign(Col + y0, Col + y1);
    std::sort(u.begin(), u.end());
    u.erase(std::unique(u.begin(), u.end()), u.end());
    for (int j = y0; j < y1; ++j) o.ecr[(size_t)j] = (int)(std::lower_bound(u.begin(), u.end(), Col[j]) - u.begin());
    o.nec[(size_t)t] = (int)u.size();
  }
  o.uxp.assign((size_t)NT + 1, 0);
  for (int64_t t = 0; t < NT; ++t) o.uxp[(size_t)t + 1] = o.uxp[(size_t)t] + o.nec[(size_t)t];
  o.ux.resize((size_t)o.uxp[(size_t)NT]);
  for (int64_t t = 0; t < NT; ++t) std::copy(used[(size_t)t].begin(), used[(size_t)t].end(), o.ux.begin() + o.uxp[(size_t)t]);
  // column groups, piece by piece in order
  o.vrp.assign((size_t)m + 1, 0);
  std::vector<int> gcount((size_t)NT, 0);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t t = 0; t < NT; ++t) {
    int g = 0;
    const int x0 = o.tcs[(size_t)(2 * t)], x1 = o.tce[(size_t)(2 * t)], ys = o.tcs[(size_t)(2 * t + 1)];
    for (int i = x0; i < x1; ++i) {
      const int ps = std::max(Rst[i], ys);
      const int cnt = Rst[i + 1] - ps;
      if (cnt > 0) {
        int cs = o.ecr[(size_t)ps];
        for (int j = 1; j < cnt; ++j)
          if (o.ecr[(size_t)(ps + j)] - cs >= nL) { g++; cs = o.ecr[(size_t)(ps + j)]; }
        g++;
      }
    }
    gcount[(size_t)t] = g;
  }
  std::vector<int64_t> gbase((size_t)NT + 1, 0);
  for (int64_t t = 0; t < NT; ++t) gbase[(size_t)t + 1] = gbase[(size_t)t] + gcount[(size_t)t];
  const int64_t ngroups = gbase[(size_t)NT];
  const double ird = ngroups > 0 ? (double)nnz / ((double)ngroups * nL) : 0.0;
  o.ird = (float)ird;
  int variant;
  if (force >= 0) variant = force;
  else if (m < 2000000) variant = (o.ird >= (float)thr) ? 0 : 1;
  else variant = 2;
  o.variant = variant;
  if (variant == 0) {
    o.cs.assign((size_t)ngroups, 0);
    o.va.assign((size_t)(ngroups * nL), T(0));
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t t = 0; t < NT; ++t) {
      int64_t g = gbase[(size_t)t];
      const int x0 = o.tcs[(size_t)(2 * t)], x1 = o.tce[(size_t)(2 * t)], ys = o.tcs[(size_t)(2 * t + 1)];
      for (int i = x0; i < x1; ++i) {
        const int ps = std::max(Rst[i], ys);
        const int cnt = Rst[i + 1] - ps;
        if (cnt > 0) {
          int cs = o.ecr[(size_t)ps];
          o.cs[(size_t)g] = cs;
          for (int j = 0; j < cnt; ++j) {
            const int e = o.ecr[(size_t)(ps + j)];
            if (e - cs >= nL) { g++; cs = e; o.cs[(size_t)g] = cs; }
            o.va[(size_t)(g * nL + (e - cs))] = Val[ps + j];
          }
          g++;
        }
        o.vrp[(size_t)i + 1] = (int)g;
      }
    }
    for (int64_t i = 0; i < m; ++i) o.vrp[(size_t)i + 1] = std::max(o.vrp[(size_t)i + 1], o.vrp[(size_t)i]);
  } else if (variant == 1) {
    std::vector<int> row_lo((size_t)NT + 1);
    for (int64_t t = 0; t <= NT; ++t) {
      int x, y;
      merge_path_host(std::min(ipt * t, items), Rst + 1, m, nnz, &x, &y);
      row_lo[(size_t)t] = x;
    }
    row_lo[(size_t)NT] = (int)m;
    std::vector<std::vector<int>> su((size_t)NT);
    std::vector<std::vector<int>> tk((size_t)NT), rb((size_t)NT), re((size_t)NT), rc((size_t)NT);
    std::vector<std::vector<T>> rv((size_t)NT);
    std::vector<int> spv((size_t)NT, 0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t t = 0; t < NT; ++t) {
      const int r0 = row_lo[(size_t)t], r1 = std::max(r0, row_lo[(size_t)t + 1]);
      std::vector<int>& u = su[(size_t)t];
      u.assign(Col + Rst[r0], Col + Rst[r1]);
      std::sort(u.begin(), u.end());
      u.erase(std::unique(u.begin(), u.end()), u.end());
      auto rank = [&](int c) { return (int)(std::lower_bound(u.begin(), u.end(), c) - u.begin()); };
      std::vector<int> shortr, longr;
      for (int r = r0; r < r1; ++r) ((Rst[r + 1] - Rst[r]) < nL ? shortr : longr).push_back(r);
      std::stable_sort(shortr.begin(), shortr.end(),
                       [&](int a, int b) { return (Rst[a + 1] - Rst[a]) > (Rst[b + 1] - Rst[b]); });
      const int64_t ngr = (int64_t)shortr.size() / nL;
      spv[(size_t)t] = (int)(ngr * nL);
      for (int64_t q = 0; q < ngr; ++q) {
        const int rl = Rst[shortr[(size_t)(q * nL)] + 1] - Rst[shortr[(size_t)(q * nL)]];
        const int base = (int)rc[(size_t)t].size();
        rc[(size_t)t].resize((size_t)(base + rl * nL), 0);
        rv[(size_t)t].resize((size_t)(base + rl * nL), T(0));
        for (int k = 0; k < nL; ++k) {
          const int r = shortr[(size_t)(q * nL + k)];
          tk[(size_t)t].push_back(r);
          rb[(size_t)t].push_back(base);
          re[(size_t)t].push_back(base + rl);
          for (int c = 0; c < Rst[r + 1] - Rst[r]; ++c) {
            rc[(size_t)t][(size_t)(base + c * nL + k)] = rank(Col[Rst[r] + c]);
            rv[(size_t)t][(size_t)(base + c * nL + k)] = Val[Rst[r] + c];
          }
        }
      }
      std::vector<int> inrow(shortr.begin() + ngr * nL, shortr.end());
      inrow.insert(inrow.end(), longr.begin(), longr.end());
      for (int r : inrow) {
        tk[(size_t)t].push_back(r);
        rb[(size_t)t].push_back((int)rc[(size_t)t].size());
        for (int k = Rst[r]; k < Rst[r + 1]; ++k) {
          rc[(size_t)t].push_back(rank(Col[k]));
          rv[(size_t)t].push_back(Val[k]);
        }
        re[(size_t)t].push_back((int)rc[(size_t)t].size());
      }
    }
    // concatenate pieces; row_begin/row_end become global offsets
    o.nec.assign((size_t)NT, 0);
    o.uxp.assign((size_t)NT + 1, 0);
    o.ux.clear();
    o.ts.assign((size_t)NT, 0);
    o.te.assign((size_t)NT, 0);
    o.spv = spv;
    o.tasks.clear(); o.rb.clear(); o.re.clear(); o.rc.clear(); o.rv.clear();
    for (int64_t t = 0; t < NT; ++t) {
      o.nec[(size_t)t] = (int)su[(size_t)t].size();
      o.ux.insert(o.ux.end(), su[(size_t)t].begin(), su[(size_t)t].end());
      o.uxp[(size_t)t + 1] = (int)o.ux.size();
      o.ts[(size_t)t] = (int)o.tasks.size();
      const int off = (int)o.rc.size();
      o.tasks.insert(o.tasks.end(), tk[(size_t)t].begin(), tk[(size_t)t].end());
      for (int v : rb[(size_t)t]) o.rb.push_back(v + off);
      for (int v : re[(size_t)t]) o.re.push_back(v + off);
      o.rc.insert(o.rc.end(), rc[(size_t)t].begin(), rc[(size_t)t].end());
      o.rv.insert(o.rv.end(), rv[(size_t)t].begin(), rv[(size_t)t].end());
      o.te[(size_t)t] = (int)o.tasks.size();
    }
  }
  o.max_nec = 0;
  for (int v : o.nec) o.max_nec = std::max(o.max_nec, v);
}

template void vnec_build_host<float>(const int*, const int*, const float*, int64_t, int64_t, int64_t, int64_t, int,
                                     int, double, VnecHost<float>&);
template void vnec_build_host<double>(const int*, const int*, const double*, int64_t, int64_t, int64_t, int64_t,
                                      int, int, double, VnecHost<double>&);

}  // namespace rvvla
