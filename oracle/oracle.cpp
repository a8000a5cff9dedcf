// oracle.cpp — CPU restatement of RVVLASparse's SpMV path (TEST INFRASTRUCTURE
// ONLY; see oracle.h for what is pinned and how).  Compiled by oracle/Makefile
// with -fno-tree-vectorize -ffp-contract=off so the plain scalar restatements
// round exactly like the reference scalar library (which is built with
// -fno-tree-vectorize and no FMA contraction on x86-64).
//
// Every function cites the reference file:line it restates.  Builders for the
// formats whose reference builder is missing cite the kernel lines that define
// the layout they must produce.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <numeric>
#include <stdexcept>
#include <type_traits>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

int dtype_size(int dt) {
  switch (dt) {
    case ORC_I32: case ORC_U32: case ORC_F32: return 4;
    case ORC_U16: return 2;
    case ORC_U8: return 1;
    default: return 8;
  }
}

struct Arr {
  std::string name;
  int dtype;
  int64_t len;
  std::vector<uint8_t> bytes;
};

struct Bundle {
  std::string fmt;
  std::vector<Arr> arrs;
  std::vector<std::pair<std::string, double>> sc;

  const Arr* find(const std::string& n) const {
    for (auto& a : arrs)
      if (a.name == n) return &a;
    return nullptr;
  }
  template <class T>
  const T* get(const std::string& n, int64_t* len = nullptr) const {
    const Arr* a = find(n);
    if (!a) throw std::runtime_error(fmt + ": missing array " + n);
    if (len) *len = a->len;
    return reinterpret_cast<const T*>(a->bytes.data());
  }
  template <class T>
  void put(const std::string& n, int dt, const std::vector<T>& v) {
    Arr a;
    a.name = n;
    a.dtype = dt;
    a.len = (int64_t)v.size();
    a.bytes.resize(v.size() * sizeof(T));
    if (!v.empty()) std::memcpy(a.bytes.data(), v.data(), a.bytes.size());
    for (auto& e : arrs)
      if (e.name == n) { e = std::move(a); return; }
    arrs.push_back(std::move(a));
  }
  void set(const std::string& n, double v) {
    for (auto& e : sc)
      if (e.first == n) { e.second = v; return; }
    sc.emplace_back(n, v);
  }
  double s(const std::string& n) const {
    for (auto& e : sc)
      if (e.first == n) return e.second;
    throw std::runtime_error(fmt + ": missing scalar " + n);
  }
  int64_t i(const std::string& n) const { return (int64_t)s(n); }
};

template <class T> constexpr int dt_of();
template <> constexpr int dt_of<float>() { return ORC_F32; }
template <> constexpr int dt_of<double>() { return ORC_F64; }

// ---------------------------------------------------------------- CSR view
template <class T>
struct Crs {
  int64_t m, n, nz;
  const int* Rst;
  const int* Col;
  const T* Val;
};

template <class T>
Crs<T> crs_view(const Bundle& b) {
  Crs<T> A;
  A.m = b.i("m");
  A.n = b.i("n");
  A.nz = b.i("nz");
  A.Rst = b.get<int>("Rst");
  A.Col = b.get<int>("Col");
  A.Val = b.get<T>("Val");
  return A;
}

int val_dtype(const Bundle& b) {
  for (auto& a : b.arrs)
    if (a.dtype == ORC_F32 || a.dtype == ORC_F64) return a.dtype;
  return (int)b.s("dtype");
}

template <class T>
Bundle* new_crs(int64_t m, int64_t n, const std::vector<int>& Rst, const std::vector<int>& Col,
                const std::vector<T>& Val) {
  auto* b = new Bundle();
  b->fmt = "crs";
  b->set("m", (double)m);
  b->set("n", (double)n);
  b->set("nz", (double)Col.size());
  b->set("dtype", dt_of<T>());
  b->put("Rst", ORC_I32, Rst);
  b->put("Col", ORC_I32, Col);
  b->put("Val", dt_of<T>(), Val);
  return b;
}

// =====================================================================
// CRS SpMV — src/scalar/spmv_mtx_crs.cpp:22-71 (row-sequential sum in index
// order, then y[i] = tmp*alpha + beta*y[i]).
// =====================================================================
template <class T>
void crs_spmv(const Crs<T>& A, T alpha, const T* b, T beta, T* y) {
  for (int64_t i = 0; i < A.m; i++) {
    T tmp = 0;
    for (int64_t j = A.Rst[i]; j < A.Rst[i + 1]; j++) tmp += A.Val[j] * b[A.Col[j]];
    y[i] = tmp * alpha + beta * y[i];
  }
}

// =====================================================================
// HCSR builder — src/scalar/crs_to_hcsr.cpp:30-135 (crs_to_HCSR), restated.
// Block classification: kind 0 empty, 1 CSR if rows*p < cnt, else 2 COO
// (:61-77); serial scans of block_ptr/row_offset with the 30-bit limit and nnz
// check (:79-91); stable scatter in source order (:97-119); in-block prefix sum
// for CSR blocks (:121-126); kind in bits 31:30 of row_offset (:130-134).
// =====================================================================
template <class T>
Bundle* build_hcsr(const Crs<T>& A, int64_t R_, int64_t C_, double bs) {
  if (R_ <= 0 || C_ <= 0) throw std::invalid_argument("crs_to_HCSR: R and C must be positive");
  const size_t R = (size_t)R_, C = (size_t)C_;
  const size_t m = (size_t)A.m, n = (size_t)A.n, nz = (size_t)A.nz;
  const size_t b_m = (m + R - 1) / R, b_n = (n + C - 1) / C;
  const size_t nblocks = b_m * b_n;
  if (b_n != 0 && nblocks / b_n != b_m) throw std::length_error("crs_to_HCSR: too many blocks");
  std::vector<int> block_ptr(nblocks + 1, 0);
  std::vector<uint32_t> row_offset(nblocks + 1, 0);
  std::vector<uint8_t> kind(nblocks, 0);
  for (size_t br = 0; br < b_m; ++br) {
    const size_t r0 = br * R, r1 = std::min(r0 + R, m);
    const size_t blk0 = br * b_n;
    int* cnt = block_ptr.data() + blk0 + 1;
    for (size_t i = r0; i < r1; ++i)
      for (size_t k = (size_t)A.Rst[i]; k < (size_t)A.Rst[i + 1]; ++k) ++cnt[(size_t)A.Col[k] / C];
    const double rows = double(r1 - r0);
    for (size_t j = 0; j < b_n; ++j) {
      const size_t c = (size_t)cnt[j];
      if (c == 0) { kind[blk0 + j] = 0; row_offset[blk0 + j + 1] = 0; }
      else if (rows * bs < double(c)) { kind[blk0 + j] = 1; row_offset[blk0 + j + 1] = (uint32_t)(r1 - r0 + 1); }
      else { kind[blk0 + j] = 2; row_offset[blk0 + j + 1] = (uint32_t)c; }
    }
  }
  size_t accNz = 0, accRows = 0;
  const size_t flagLimit = (size_t(1) << 30) - 1;
  for (size_t b = 1; b <= nblocks; ++b) {
    accNz += (size_t)block_ptr[b];
    accRows += (size_t)row_offset[b];
    block_ptr[b] = (int)accNz;
    row_offset[b] = (uint32_t)accRows;
  }
  if (accRows > flagLimit)
    throw std::length_error("crs_to_HCSR: row_ptr has " + std::to_string(accRows) +
                            " entries, does not fit the 30-bit row_offset field");
  if (accNz != nz) throw std::logic_error("crs_to_HCSR: nnz mismatch");
  std::vector<uint16_t> col_idx(nz);
  std::vector<T> values(nz);
  std::vector<uint32_t> row_ptr(accRows, 0);
  std::vector<size_t> pos(b_n);
  for (size_t br = 0; br < b_m; ++br) {
    const size_t r0 = br * R, r1 = std::min(r0 + R, m);
    const size_t blk0 = br * b_n;
    for (size_t j = 0; j < b_n; ++j) pos[j] = (size_t)block_ptr[blk0 + j];
    for (size_t i = r0; i < r1; ++i) {
      const size_t li = i - r0;
      for (size_t k = (size_t)A.Rst[i]; k < (size_t)A.Rst[i + 1]; ++k) {
        const size_t col = (size_t)A.Col[k];
        const size_t j = col / C, blk = blk0 + j;
        const size_t p = pos[j]++;
        col_idx[p] = (uint16_t)(col - j * C);
        values[p] = A.Val[k];
        const size_t ro = (size_t)row_offset[blk];
        if (kind[blk] == 1) ++row_ptr[ro + li + 1];
        else row_ptr[ro + (p - (size_t)block_ptr[blk])] = (uint32_t)li;
      }
    }
    for (size_t j = 0; j < b_n; ++j) {
      const size_t blk = blk0 + j;
      if (kind[blk] != 1) continue;
      uint32_t* rp = row_ptr.data() + (size_t)row_offset[blk];
      for (size_t li = 0; li < r1 - r0; ++li) rp[li + 1] += rp[li];
    }
  }
  for (size_t b = 0; b < nblocks; ++b) row_offset[b] |= (uint32_t)kind[b] << 30;
  auto* out = new Bundle();
  out->fmt = "hcsr";
  out->set("R", (double)R); out->set("C", (double)C);
  out->set("m", (double)m); out->set("n", (double)n); out->set("nz", (double)nz);
  out->set("b_m", (double)b_m); out->set("b_n", (double)b_n);
  out->set("dtype", dt_of<T>());
  out->put("block_ptr", ORC_I32, block_ptr);
  out->put("row_offset", ORC_U32, row_offset);
  out->put("row_ptr", ORC_U32, row_ptr);
  out->put("col_idx", ORC_U16, col_idx);
  out->put("values", dt_of<T>(), values);
  return out;
}

// HCSR SpMV — src/scalar/spmv_mtx_hcsr.cpp:22-102 (per block-row: y *= beta,
// then every column block: CSR kind -> y[i] += alpha*sum, other kinds -> COO
// y[row_ptr[k]] += alpha*v*b).
template <class T>
void hcsr_spmv(const Bundle& H, T alpha, const T* b, T beta, T* y) {
  const int64_t R = H.i("R"), C = H.i("C"), m = H.i("m"), n = H.i("n"), b_n = H.i("b_n");
  const int* block_ptr = H.get<int>("block_ptr");
  const uint32_t* row_offset = H.get<uint32_t>("row_offset");
  const uint32_t* row_ptr = H.get<uint32_t>("row_ptr");
  const uint16_t* col_idx = H.get<uint16_t>("col_idx");
  const T* values = H.get<T>("values");
  for (int64_t i = 0; i < m; i += R) {
    int64_t maxr = std::min(R, m - i);
    for (int64_t r = 0; r < maxr; ++r) y[i + r] *= beta;
    for (int64_t j = 0; j < n; j += C) {
      int64_t block = j / C + (i / R) * b_n;
      int64_t bptr = block_ptr[block];
      uint32_t rof = row_offset[block];
      uint32_t key = rof >> 30;
      rof &= 0x3FFFFFFFu;
      int64_t nzb = block_ptr[block + 1] - bptr;
      const uint32_t* rp = row_ptr + rof;
      const uint16_t* ci = col_idx + bptr;
      const T* vv = values + bptr;
      const T* bb = b + j;
      T* yy = y + i;
      if (key == 1) {
        for (int64_t r = 0; r < maxr; ++r) {
          T tmp = 0;
          for (int64_t q = rp[r]; q < (int64_t)rp[r + 1]; ++q) tmp += vv[q] * bb[ci[q]];
          yy[r] += alpha * tmp;
        }
      } else {
        for (int64_t q = 0; q < nzb; ++q) yy[rp[q]] += alpha * vv[q] * bb[ci[q]];
      }
    }
  }
}

// =====================================================================
// SELL-C-sigma builder (no reference builder).  Layout as read by
// src/scalar/spmv_mtx_sell_c_sigma.cpp:52-98 and src/rvv/...:40-88:
//   slice i: height vBs[i] (C, last one shorter), width vCl[i] (longest row),
//   start vCs[i], first sorted row vSBs[i] = i*C; element (k, j) at
//   vCs[i] + j*vBs[i] + k (column-major in the slice); vPerm[sorted] = row.
// Rows are sorted by length, descending, inside windows of sigma rows (stable:
// ties keep source order).  Padding: value 0, column 0.
// =====================================================================
template <class T>
Bundle* build_sell(const Crs<T>& A, int64_t C, int64_t sigma) {
  if (C <= 0) throw std::invalid_argument("SELL: C must be positive");
  if (sigma <= 0) sigma = 1;
  const int64_t m = A.m;
  std::vector<uint32_t> perm((size_t)m);
  std::iota(perm.begin(), perm.end(), 0u);
  auto len = [&](uint32_t r) { return (int64_t)A.Rst[r + 1] - A.Rst[r]; };
  for (int64_t w0 = 0; w0 < m; w0 += sigma) {
    int64_t w1 = std::min(m, w0 + sigma);
    std::stable_sort(perm.begin() + w0, perm.begin() + w1,
                     [&](uint32_t a, uint32_t b) { return len(a) > len(b); });
  }
  const int64_t cnt_b = (m + C - 1) / C;
  std::vector<int> vCl((size_t)cnt_b), vCs((size_t)cnt_b), vBs((size_t)cnt_b), vSBs((size_t)cnt_b);
  int64_t off = 0;
  for (int64_t s = 0; s < cnt_b; ++s) {
    int64_t r0 = s * C, r1 = std::min(m, r0 + C);
    int64_t w = 0;
    for (int64_t r = r0; r < r1; ++r) w = std::max(w, len(perm[(size_t)r]));
    vCl[(size_t)s] = (int)w;
    vBs[(size_t)s] = (int)(r1 - r0);
    vSBs[(size_t)s] = (int)r0;
    vCs[(size_t)s] = (int)off;
    off += w * (r1 - r0);
  }
  if (off > INT32_MAX) throw std::length_error("SELL: padded size exceeds int32 offsets");
  std::vector<uint32_t> vCol((size_t)off, 0u);
  std::vector<T> vVal((size_t)off, T(0));
  for (int64_t s = 0; s < cnt_b; ++s) {
    for (int64_t k = 0; k < vBs[(size_t)s]; ++k) {
      uint32_t row = perm[(size_t)(vSBs[(size_t)s] + k)];
      int64_t L = len(row);
      for (int64_t j = 0; j < L; ++j) {
        int64_t p = vCs[(size_t)s] + j * vBs[(size_t)s] + k;
        vCol[(size_t)p] = (uint32_t)A.Col[A.Rst[row] + j];
        vVal[(size_t)p] = A.Val[A.Rst[row] + j];
      }
    }
  }
  auto* out = new Bundle();
  out->fmt = "sell";
  out->set("m", (double)m); out->set("n", (double)A.n); out->set("cnt_b", (double)cnt_b);
  out->set("nz", (double)A.nz); out->set("C", (double)C); out->set("Sigma", (double)sigma);
  out->set("dtype", dt_of<T>());
  out->put("vCl", ORC_I32, vCl); out->put("vCs", ORC_I32, vCs);
  out->put("vBs", ORC_I32, vBs); out->put("vSBs", ORC_I32, vSBs);
  out->put("vCol", ORC_U32, vCol); out->put("vPerm", ORC_U32, perm);
  out->put("vVal", dt_of<T>(), vVal);
  return out;
}

// SELL SpMV, three stages — src/scalar/spmv_mtx_sell_c_sigma.cpp:22-149.
template <class T>
void sell_spmv(const Bundle& S, T alpha, const T* b, T beta, T* y, int stage) {
  const int64_t m = S.i("m"), cnt_b = S.i("cnt_b");
  const uint32_t* perm = S.get<uint32_t>("vPerm");
  if (stage == 0 || stage == 3) {  // PREPARATION :22-49 — y := y[perm]
    std::vector<T> t((size_t)m);
    for (int64_t i = 0; i < m; i++) t[(size_t)i] = y[perm[i]];
    for (int64_t i = 0; i < m; i++) y[i] = t[(size_t)i];
  }
  if (stage == 1 || stage == 3) {  // MULT :52-98
    const int* Cl = S.get<int>("vCl");
    const int* Cs = S.get<int>("vCs");
    const int* Bs = S.get<int>("vBs");
    const int* SBs = S.get<int>("vSBs");
    const uint32_t* Col = S.get<uint32_t>("vCol");
    const T* Val = S.get<T>("vVal");
    std::vector<T> yt(cnt_b > 0 ? (size_t)Bs[0] : 0);
    for (int64_t i = 0; i < cnt_b; i++) {
      int64_t cur = SBs[i];
      for (int64_t k = 0; k < Bs[i]; k++) yt[(size_t)k] = 0;
      for (int64_t j = 0; j < Cl[i]; j++)
        for (int64_t k = 0; k < Bs[i]; k++)
          yt[(size_t)k] += Val[Cs[i] + j * Bs[i] + k] * b[Col[Cs[i] + j * Bs[i] + k]];
      for (int64_t k = 0; k < Bs[i]; k++) y[cur + k] = yt[(size_t)k] * alpha + beta * y[cur + k];
    }
  }
  if (stage == 2 || stage == 3) {  // GET_RESULTS :100-127 — y[perm] := y
    std::vector<T> t(y, y + m);
    for (int64_t i = 0; i < m; i++) y[perm[i]] = t[(size_t)i];
  }
}

// =====================================================================
// CSR5 builder (asCSR5 is declared at include/CSR5.h:61-65 but never
// defined).  The layout is the one src/rvv/spmv_mtx_csr5.cpp decodes:
//   * tile t (t < p-1) holds nnz [t*w*s, (t+1)*w*s) transposed: CSR element
//     tile_start + l*sigma + i sits at tile_start + i*omega + l (:147-151,
//     :197-203);
//   * tile_pointer[t] = row holding the tile's first element, bit 31 set when
//     the tile needs the empty-row map (:156-167);
//   * per lane, tile_desc_len dwords at tile*omega*tdl + d*omega + l: dword 0
//     holds y_offset (top bit_y_offset bits), seg_offset (next bit_seg_offset
//     bits) and the row-start flags of steps 0.., MSB first; later dwords hold
//     32 flags each (:176-245);
//   * y_offset[l] = row starts in lanes < l, not counting tile element 0
//     (rows are written to y[tile_first_row + 1 + y_offset], :227-236);
//   * seg_offset[l] = number of following lanes with no row start (:256-262);
//   * tile_empty_offset[ptr + k] = (row of the k-th row start) -
//     tile_first_row - 1, for tiles flagged in bit 31 (:226-229);
//   * the last (possibly partial) tile stays in CSR order and is handled by
//     the tail kernel from row tail_tile_start (:337-365).
// Bit widths follow Liu & Vinter's CSR5: bits(omega*sigma), bits(omega).
// =====================================================================
int bits_for(int64_t v) {
  int r = 0;
  while (v) { r++; v >>= 1; }
  return r;
}

int64_t row_of(const int* Rst, int64_t m, int64_t e) {
  // largest r in [0, m] with Rst[r] <= e
  return (int64_t)(std::upper_bound(Rst, Rst + m + 1, (int)e) - Rst) - 1;
}

template <class T>
Bundle* build_csr5(const Crs<T>& A, int64_t omega, int64_t sigma) {
  if (omega <= 0 || sigma <= 0) throw std::invalid_argument("CSR5: omega and sigma must be positive");
  const int64_t m = A.m, nnz = A.nz, ws = omega * sigma;
  int64_t p = (nnz + ws - 1) / ws;
  if (p < 1) p = 1;
  const int by = bits_for(ws), bsg = bits_for(omega);
  if (by + bsg >= 32) throw std::invalid_argument("CSR5: omega*sigma too large");
  const int flag0 = 32 - by - bsg;
  const int64_t tdl = (by + bsg + sigma + 31) / 32;
  std::vector<uint32_t> tile_ptr((size_t)p + 1);
  for (int64_t t = 0; t <= p; ++t) {
    int64_t bnd = std::min(t * ws, nnz);
    tile_ptr[(size_t)t] = (uint32_t)row_of(A.Rst, m, bnd);
  }
  // row-start marker: first element of a non-empty row
  std::vector<uint8_t> is_start((size_t)nnz, 0);
  std::vector<int> start_row((size_t)nnz, -1);
  for (int64_t r = 0; r < m; ++r)
    if (A.Rst[r + 1] > A.Rst[r]) { is_start[(size_t)A.Rst[r]] = 1; start_row[(size_t)A.Rst[r]] = (int)r; }
  const int64_t nfull = p - 1;
  std::vector<uint32_t> desc((size_t)(nfull * omega * tdl), 0u);
  std::vector<uint32_t> eo_ptr((size_t)p, 0u);
  std::vector<uint32_t> eo;
  for (int64_t t = 0; t < nfull; ++t) {
    const int64_t s0 = t * ws;
    const int64_t first = tile_ptr[(size_t)t];
    std::vector<int> lane_has(omega, 0);
    for (int64_t l = 0; l < omega; ++l)
      for (int64_t i = 0; i < sigma; ++i)
        if (is_start[(size_t)(s0 + l * sigma + i)]) lane_has[(size_t)l] = 1;
    int64_t yoff = 0;
    bool identity = true;
    std::vector<uint32_t> rows_k;
    for (int64_t l = 0; l < omega; ++l) {
      int64_t seg = 0;
      while (l + seg + 1 < omega && !lane_has[(size_t)(l + seg + 1)]) seg++;
      uint32_t* d = desc.data() + (size_t)(t * omega * tdl);
      d[l] = ((uint32_t)yoff << (32 - by)) | ((uint32_t)seg << (32 - by - bsg));
      for (int64_t i = 0; i < sigma; ++i) {
        int64_t e = l * sigma + i;
        if (!is_start[(size_t)(s0 + e)]) continue;
        int64_t dw, bit;
        if (i < flag0) { dw = 0; bit = 31 - by - bsg - i; }
        else { dw = 1 + (i - flag0) / 32; bit = 31 - (i - flag0) % 32; }
        d[dw * omega + l] |= (uint32_t)1u << bit;
        if (e == 0) continue;  // tile element 0 belongs to tile_first_row
        int64_t row = start_row[(size_t)(s0 + e)];
        if (row != first + 1 + yoff) identity = false;
        rows_k.push_back((uint32_t)(row - first - 1));
        yoff++;
      }
    }
    eo_ptr[(size_t)t] = (uint32_t)eo.size();
    if (!identity) {
      tile_ptr[(size_t)t] |= 0x80000000u;
      eo.insert(eo.end(), rows_k.begin(), rows_k.end());
    }
  }
  if (nfull < p) eo_ptr[(size_t)(p - 1)] = (uint32_t)eo.size();
  std::vector<uint32_t> col((size_t)nnz);
  std::vector<T> val((size_t)nnz);
  for (int64_t t = 0; t < nfull; ++t)
    for (int64_t l = 0; l < omega; ++l)
      for (int64_t i = 0; i < sigma; ++i) {
        int64_t src = t * ws + l * sigma + i, dst = t * ws + i * omega + l;
        col[(size_t)dst] = (uint32_t)A.Col[src];
        val[(size_t)dst] = A.Val[src];
      }
  for (int64_t k = nfull * ws; k < nnz; ++k) { col[(size_t)k] = (uint32_t)A.Col[k]; val[(size_t)k] = A.Val[k]; }
  std::vector<int> rp(A.Rst, A.Rst + m + 1);
  auto* out = new Bundle();
  out->fmt = "csr5";
  out->set("m", (double)m); out->set("n", (double)A.n); out->set("nnz", (double)nnz);
  out->set("bit_y_offset", by); out->set("bit_seg_offset", bsg); out->set("tile_desc_len", (double)tdl);
  out->set("tail_tile_start", (double)(tile_ptr[(size_t)(p - 1)] & 0x7FFFFFFFu));
  out->set("p", (double)p); out->set("omega", (double)omega); out->set("sigma", (double)sigma);
  out->set("num_offsets", (double)eo.size());
  out->set("dtype", dt_of<T>());
  out->put("csr_row_pointer", ORC_I32, rp);
  out->put("csr_column_index", ORC_U32, col);
  out->put("csr_value", dt_of<T>(), val);
  out->put("tile_pointer", ORC_U32, tile_ptr);
  out->put("tile_descriptor", ORC_U32, desc);
  out->put("tile_empty_offset_pointer", ORC_U32, eo_ptr);
  out->put("tile_empty_offset", ORC_U32, eo);
  return out;
}

// CSR5 SpMV — restates src/rvv/spmv_mtx_csr5.cpp:33-365 lane by lane, run as a
// single thread (so every tile-first-row partial goes straight to y; the
// calibrator of :318-335 only serialises the per-thread first rows).
template <class T>
void csr5_spmv(const Bundle& B, T alpha, const T* x, T beta, T* y) {
  const int64_t m = B.i("m"), p = B.i("p"), omega = B.i("omega"), sigma = B.i("sigma");
  const int by = (int)B.i("bit_y_offset"), bsg = (int)B.i("bit_seg_offset");
  const int64_t tdl = B.i("tile_desc_len"), tail = B.i("tail_tile_start");
  const int* rp = B.get<int>("csr_row_pointer");
  const uint32_t* ci = B.get<uint32_t>("csr_column_index");
  const T* cv = B.get<T>("csr_value");
  const uint32_t* tp = B.get<uint32_t>("tile_pointer");
  const uint32_t* td = B.get<uint32_t>("tile_descriptor");
  const uint32_t* teop = B.get<uint32_t>("tile_empty_offset_pointer");
  const uint32_t* teo = B.get<uint32_t>("tile_empty_offset");
  for (int64_t i = 0; i < m; ++i) y[i] *= beta;  // :513-517
  const int64_t W = omega;
  std::vector<T> sum(W), first_sum(W), last_sum(W), sh(W), S(W);
  std::vector<uint32_t> yoff(W), segoff(W), cur(W), stopc(W);
  std::vector<uint8_t> start(W), incol(W), lb(W);
  for (int64_t t = 0; t + 1 < p; ++t) {  // :139 (tiles 0..p-2)
    const T* val = cv + t * omega * sigma;
    const uint32_t* col = ci + t * omega * sigma;
    const uint32_t* d = td + t * omega * tdl;
    uint32_t first = tp[t];
    const uint32_t last = tp[t + 1] & 0x7FFFFFFFu;
    if (first == last) {  // :154-164 simple loop: whole tile in one row
      T s = 0;
      for (int64_t e = 0; e < omega * sigma; ++e) s += val[e] * x[col[e]];
      s *= alpha;
      y[first] += s;
      continue;
    }
    const bool empty = (first >> 31) & 1u;  // :166-170
    first &= 0x7FFFFFFFu;
    T* ylocal = y + first + 1;
    const uint32_t optr = empty ? teop[t] : 0;
    auto yidx = [&](uint32_t k) { return empty ? teo[optr + k] : k; };
    for (int64_t l = 0; l < W; ++l) {  // :175-203
      uint32_t d0 = d[l];
      yoff[l] = d0 >> (32 - by);
      segoff[l] = (d0 << by) >> (32 - bsg);
      cur[l] = d0 << (by + bsg);
      lb[l] = (cur[l] >> 31) & 1u;
      if (l == 0) lb[l] = 1;
      start[l] = !lb[l];
      incol[l] = lb[l] && l != 0;
      first_sum[l] = 0;
      stopc[l] = 0;
      sum[l] = val[l] * x[col[l]];
    }
    int ly = 0;
    for (int64_t i = 1; i < sigma; ++i) {  // :205-248
      int64_t norm_i = i - (32 - by - bsg);
      if (norm_i % 32 == 0) {
        ly++;
        for (int64_t l = 0; l < W; ++l) cur[l] = d[ly * omega + l];
      }
      int64_t ni = (ly == 0) ? i : norm_i % 32;
      int64_t off = 31 - ni;
      bool any = false;
      for (int64_t l = 0; l < W; ++l) { lb[l] = (cur[l] >> off) & 1u; any |= lb[l]; }
      if (any) {
        for (int64_t l = 0; l < W; ++l) {
          if (!lb[l]) continue;
          if (incol[l]) {  // green segment: a full row that started in this lane
            ylocal[yidx(yoff[l])] += alpha * sum[l];
            yoff[l]++;
          } else {  // red segment: this lane's leading part
            first_sum[l] = sum[l];
          }
          sum[l] = 0;
          incol[l] = 1;
          stopc[l]++;
        }
      }
      for (int64_t l = 0; l < W; ++l) sum[l] += val[i * omega + l] * x[col[i * omega + l]];
    }
    for (int64_t l = 0; l < W; ++l) {  // :250-276
      if (!incol[l]) first_sum[l] = sum[l];
      last_sum[l] = sum[l];
    }
    for (int64_t l = 0; l < W; ++l) {
      T lead_next = (l + 1 < W && start[l + 1]) ? first_sum[l + 1] : T(0);
      sh[l] = lead_next;
    }
    for (int64_t l = 0; l < W; ++l) {
      // sum of sh[l .. l+seg_offset[l]] (the slide-up scan differenced at :262-264)
      T acc = 0;
      int64_t e = std::min<int64_t>(W - 1, l + (int64_t)segoff[l]);
      for (int64_t k = l; k <= e; ++k) acc += sh[k];
      S[l] = acc;
    }
    for (int64_t l = 0; l < W; ++l)
      if ((uint32_t)start[l] <= stopc[l]) last_sum[l] += S[l];  // :265-266
    for (int64_t l = 0; l < W; ++l)
      if (incol[l]) ylocal[yidx(yoff[l])] += alpha * last_sum[l];  // :268-274
    T add = incol[0] ? first_sum[0] : last_sum[0];  // :276-278
    add *= alpha;
    y[first] += add;
  }
  // tail kernel :337-365
  for (int64_t row = tail; row < m; ++row) {
    int64_t s = (row == tail) ? (p - 1) * omega * sigma : rp[row];
    T acc = 0;
    for (int64_t k = s; k < rp[row + 1]; ++k) acc += cv[k] * x[ci[k]];
    acc *= alpha;
    y[row] += acc;
  }
}

// =====================================================================
// LAV builder (no reference builder).  Layout as read by
// src/scalar/spmv_mtx_lav.cpp:36-79:
//   segment s, chunk c (SIMD_Lanes rows out_order[(c + chunk_count*s)*L + i]);
//   chunk steps [chunk_offsets[(chunk_count+1)*s + c], ...[+1]) relative to
//   segment_ptr[s]; steps before chunk_offsets_full_mask[s*chunk_count + c]
//   use all L lanes, later steps use mask[step] lanes (a prefix);
//   val/col_id at (segment_ptr[s] + step)*L + i; the rest in sparse_part (CRS),
//   which applies beta to every row.
// Dense columns: the densest columns holding >= (1-T) of the nonzeros (ties by
// column index), cut into segments of segment_len columns in density order.
// Rows: one global chunking (rows by dense count, descending, stable), and in
// each segment the rows of a chunk are ordered by their count in that segment
// (descending, stable) so active lanes form a prefix.  Pad slots of the last
// chunk hold row index m-1 and are never active.
// =====================================================================
template <class T>
Bundle* build_lav(const Crs<T>& A, int64_t L, double Tthr, int64_t seglen) {
  if (L <= 0 || seglen <= 0) throw std::invalid_argument("LAV: SIMD_Lanes and segment_len must be positive");
  const int64_t m = A.m, n = A.n, nz = A.nz;
  std::vector<int64_t> ccount((size_t)n, 0);
  for (int64_t k = 0; k < nz; ++k) ccount[(size_t)A.Col[k]]++;
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
  const int64_t chunk_count = (m + L - 1) / L;
  // per-row dense counts
  std::vector<int64_t> dcount((size_t)m, 0);
  std::vector<int> sRst((size_t)m + 1, 0);
  for (int64_t r = 0; r < m; ++r)
    for (int64_t k = A.Rst[r]; k < A.Rst[r + 1]; ++k) {
      if (seg_of[(size_t)A.Col[k]] >= 0) dcount[(size_t)r]++;
      else sRst[(size_t)r + 1]++;
    }
  for (int64_t r = 0; r < m; ++r) sRst[(size_t)r + 1] += sRst[(size_t)r];
  std::vector<int> sCol((size_t)sRst[(size_t)m]);
  std::vector<T> sVal((size_t)sRst[(size_t)m]);
  for (int64_t r = 0, q = 0; r < m; ++r)
    for (int64_t k = A.Rst[r]; k < A.Rst[r + 1]; ++k)
      if (seg_of[(size_t)A.Col[k]] < 0) { sCol[(size_t)q] = A.Col[k]; sVal[(size_t)q] = A.Val[k]; q++; }
  std::vector<uint32_t> gorder((size_t)m);
  std::iota(gorder.begin(), gorder.end(), 0u);
  std::stable_sort(gorder.begin(), gorder.end(), [&](uint32_t a, uint32_t b) { return dcount[a] > dcount[b]; });
  std::vector<int> chunk_offsets((size_t)((chunk_count + 1) * nseg), 0);
  std::vector<int> chunk_full((size_t)(chunk_count * nseg), 0);
  std::vector<uint64_t> segment_ptr((size_t)nseg + 1, 0);
  std::vector<uint32_t> out_order((size_t)(nseg * chunk_count * L), (uint32_t)(m > 0 ? m - 1 : 0));
  std::vector<uint16_t> mask;
  std::vector<T> val;
  std::vector<uint32_t> col_id;
  // each row's dense entries ordered by segment (stable: column order inside
  // a segment); cur[r] = the row's first entry of the current segment
  std::vector<int64_t> dptr((size_t)m + 1, 0), cur((size_t)m);
  std::vector<int> dk;
  for (int64_t r = 0; r < m; ++r) {
    const size_t b = dk.size();
    for (int64_t k = A.Rst[r]; k < A.Rst[r + 1]; ++k)
      if (seg_of[(size_t)A.Col[k]] >= 0) dk.push_back((int)k);
    std::stable_sort(dk.begin() + (std::ptrdiff_t)b, dk.end(),
                     [&](int a, int c) { return seg_of[(size_t)A.Col[a]] < seg_of[(size_t)A.Col[c]]; });
    dptr[(size_t)r + 1] = (int64_t)dk.size();
    cur[(size_t)r] = dptr[(size_t)r];
  }
  std::vector<int64_t> scount((size_t)m);
  for (int64_t s = 0; s < nseg; ++s) {
    for (int64_t r = 0; r < m; ++r) {
      int64_t c = 0;
      while (cur[(size_t)r] + c < dptr[(size_t)r + 1] && seg_of[(size_t)A.Col[dk[(size_t)(cur[(size_t)r] + c)]]] == s) c++;
      scount[(size_t)r] = c;
    }
    int64_t step = 0;
    for (int64_t c = 0; c < chunk_count; ++c) {
      int64_t r0 = c * L, r1 = std::min(m, r0 + L);
      std::vector<uint32_t> rows(gorder.begin() + r0, gorder.begin() + r1);
      std::stable_sort(rows.begin(), rows.end(), [&](uint32_t a, uint32_t b) { return scount[a] > scount[b]; });
      for (size_t i = 0; i < rows.size(); ++i) out_order[(size_t)((c + chunk_count * s) * L) + i] = rows[i];
      int64_t maxc = rows.empty() ? 0 : scount[rows[0]];
      int64_t minc = ((int64_t)rows.size() < L) ? 0 : scount[rows.back()];
      chunk_offsets[(size_t)((chunk_count + 1) * s + c)] = (int)step;
      chunk_full[(size_t)(s * chunk_count + c)] = (int)(step + minc);
      std::vector<std::vector<std::pair<uint32_t, T>>> ent(rows.size());
      for (size_t i = 0; i < rows.size(); ++i)
        for (int64_t q = 0; q < scount[rows[i]]; ++q) {
          const int k = dk[(size_t)(cur[rows[i]] + q)];
          ent[i].emplace_back((uint32_t)A.Col[k], A.Val[k]);
        }
      for (int64_t q = 0; q < maxc; ++q) {
        uint16_t active = 0;
        for (int64_t i = 0; i < L; ++i) {
          bool act = i < (int64_t)rows.size() && (int64_t)ent[(size_t)i].size() > q;
          if (act) active++;
          col_id.push_back(act ? ent[(size_t)i][(size_t)q].first : 0u);
          val.push_back(act ? ent[(size_t)i][(size_t)q].second : T(0));
        }
        mask.push_back(active);
      }
      step += maxc;
    }
    for (int64_t r = 0; r < m; ++r) cur[(size_t)r] += scount[(size_t)r];
    chunk_offsets[(size_t)((chunk_count + 1) * s + chunk_count)] = (int)step;
    segment_ptr[(size_t)s + 1] = segment_ptr[(size_t)s] + (uint64_t)step;
  }
  auto* out = new Bundle();
  out->fmt = "lav";
  out->set("SIMD_Lanes", (double)L); out->set("m", (double)m); out->set("n", (double)n);
  out->set("nz", (double)nz); out->set("segment_count", (double)nseg);
  out->set("chunk_count", (double)chunk_count); out->set("T", Tthr);
  out->set("segment_len", (double)seglen); out->set("dtype", dt_of<T>());
  out->set("sparse_nz", (double)sCol.size());
  out->put("chunk_offsets", ORC_I32, chunk_offsets);
  out->put("chunk_offsets_full_mask", ORC_I32, chunk_full);
  out->put("segment_ptr", ORC_U64, segment_ptr);
  out->put("out_order", ORC_U32, out_order);
  out->put("mask", ORC_U16, mask);
  out->put("val", dt_of<T>(), val);
  out->put("col_id", ORC_U32, col_id);
  out->put("sp_Rst", ORC_I32, sRst);
  out->put("sp_Col", ORC_I32, sCol);
  out->put("sp_Val", dt_of<T>(), sVal);
  return out;
}

// LAV SpMV — src/scalar/spmv_mtx_lav.cpp:23-82 (CRS on sparse_part with beta,
// then y[out_order] += alpha*val*b per element, segment by segment).
template <class T>
void lav_spmv(const Bundle& B, T alpha, const T* b, T beta, T* y) {
  Crs<T> sp{B.i("m"), B.i("n"), B.i("sparse_nz"), B.get<int>("sp_Rst"), B.get<int>("sp_Col"), B.get<T>("sp_Val")};
  crs_spmv(sp, alpha, b, beta, y);
  const int64_t L = B.i("SIMD_Lanes"), nseg = B.i("segment_count"), cc = B.i("chunk_count");
  const int* co = B.get<int>("chunk_offsets");
  const int* cf = B.get<int>("chunk_offsets_full_mask");
  const uint64_t* sp_ = B.get<uint64_t>("segment_ptr");
  const uint32_t* oo = B.get<uint32_t>("out_order");
  const uint16_t* mk = B.get<uint16_t>("mask");
  const T* v = B.get<T>("val");
  const uint32_t* ci = B.get<uint32_t>("col_id");
  for (int64_t s = 0; s < nseg; ++s) {
    const T* cv = v + sp_[s] * L;
    const uint32_t* cc_ = ci + sp_[s] * L;
    const uint16_t* cm = mk + sp_[s];
    const int64_t sh = (cc + 1) * s;
    for (int64_t c = 0; c < cc; ++c) {
      int64_t end = co[sh + c + 1], fe = cf[s * cc + c];
      for (int64_t lane = co[sh + c]; lane < fe; ++lane)
        for (int64_t i = 0; i < L; ++i)
          y[oo[i + (c + cc * s) * L]] += alpha * cv[lane * L + i] * b[cc_[lane * L + i]];
      for (int64_t lane = fe; lane < end; ++lane) {
        uint16_t bs = cm[lane];
        for (int64_t i = 0; i < bs; ++i)
          y[oo[i + (c + cc * s) * L]] += alpha * cv[lane * L + i] * b[cc_[lane * L + i]];
      }
    }
  }
}

// =====================================================================
// VNEC — include/VNEC.h:78-227 and src/rvv/spmv_mtx_vnec.cpp:42-586.
// Merge-path partition of (row ends, nz indices) into NUM_THREADS pieces
// (VNEC.h:89-100, MergePathDivide :42-71); x compaction per thread
// (VNEC.h:104-140); nLanes-wide column groups per row (VNEC.h:147-177);
// IRD = nnz / (groups*nLanes); variant L if m >= 2,000,000, else D if
// IRD >= IRD_thr, else S (VNEC.h:218-226; thresholds SpB_mxv_VNEC.h:22-25).
// The reference builds no D or S structure; here:
//   D: val_align[g*nLanes + (ecr - col_start[g])] = value, zero elsewhere;
//      use_x_indices[tid] = the thread's used columns, ascending.
//   S: each thread owns whole rows (contiguous range balanced by nnz); rows
//      shorter than nLanes go to cross-row groups of nLanes rows (sorted by
//      length, descending, stable; padded with value 0 / compacted column 0),
//      the remaining rows are in-row; every row of the matrix is in exactly one
//      task so beta reaches every row.
// =====================================================================
void merge_path(int64_t diagonal, const int* a, int64_t a_len, int64_t b_len, int64_t* x, int64_t* yv) {
  // MergePathDivide with b = 0..b_len-1 (nz_indices)
  int64_t x_min = std::max<int64_t>(diagonal - b_len, 0);
  int64_t x_max = std::min<int64_t>(diagonal, a_len);
  while (x_min < x_max) {
    int64_t pivot = (x_min + x_max) >> 1;
    if ((int64_t)a[pivot] <= diagonal - pivot - 1) x_min = pivot + 1;
    else x_max = pivot;
  }
  *x = std::min(x_min, a_len);
  *yv = diagonal - x_min;
}

template <class T>
Bundle* build_vnec(const Crs<T>& A, int64_t NT, int64_t force) {
  if (NT <= 0) throw std::invalid_argument("VNEC: NUM_THREADS must be positive");
  const int64_t m = A.m, n = A.n, nnz = A.nz;
  const int nL = std::is_same<T, float>::value ? 16 : 8;  // SpB_mxv_VNEC.h:22-23
  const double thr = std::is_same<T, float>::value ? 0.437 : 0.477;
  const int64_t items = nnz + m;
  const int64_t ipt = (items + NT - 1) / NT;
  std::vector<int> tcs((size_t)NT * 2), tce((size_t)NT * 2);
  for (int64_t t = 0; t < NT; ++t) {
    int64_t d0 = std::min(ipt * t, items), d1 = std::min(d0 + ipt, items);
    int64_t x, yv;
    merge_path(d0, A.Rst + 1, m, nnz, &x, &yv);
    tcs[(size_t)(2 * t)] = (int)x; tcs[(size_t)(2 * t + 1)] = (int)yv;
    merge_path(d1, A.Rst + 1, m, nnz, &x, &yv);
    tce[(size_t)(2 * t)] = (int)x; tce[(size_t)(2 * t + 1)] = (int)yv;
  }
  // per-thread compaction (merge-path ranges)
  std::vector<int> ecr((size_t)nnz, 0), nec((size_t)NT, 0), ux_ptr((size_t)NT + 1, 0), ux;
  std::vector<int> mark((size_t)n, -1), rank((size_t)n, 0);  // rank: column -> compacted index
  for (int64_t t = 0; t < NT; ++t) {
    int64_t y0 = tcs[(size_t)(2 * t + 1)], y1 = tce[(size_t)(2 * t + 1)];
    std::vector<int> used;
    for (int64_t j = y0; j < y1; ++j)
      if (mark[(size_t)A.Col[j]] != (int)t) { mark[(size_t)A.Col[j]] = (int)t; used.push_back(A.Col[j]); }
    std::sort(used.begin(), used.end());
    for (size_t k = 0; k < used.size(); ++k) rank[(size_t)used[k]] = (int)k;
    for (int64_t j = y0; j < y1; ++j) ecr[(size_t)j] = rank[(size_t)A.Col[j]];
    nec[(size_t)t] = (int)used.size();
    ux.insert(ux.end(), used.begin(), used.end());
    ux_ptr[(size_t)t + 1] = (int)ux.size();
  }
  // column groups (VNEC.h:147-177, done sequentially)
  std::vector<int> v_row_ptr((size_t)m + 1, 0), col_start;
  std::vector<T> val_align;
  int64_t g = 0;
  for (int64_t t = 0; t < NT; ++t) {
    int64_t x0 = tcs[(size_t)(2 * t)], x1 = tce[(size_t)(2 * t)], ys = tcs[(size_t)(2 * t + 1)];
    for (int64_t i = x0; i < x1; ++i) {
      int64_t ps = std::max<int64_t>(A.Rst[i], ys);
      int64_t cnt = A.Rst[i + 1] - ps;
      if (cnt > 0) {
        col_start.push_back(ecr[(size_t)ps]);
        val_align.resize(val_align.size() + nL, T(0));
        val_align[(size_t)(g * nL)] = A.Val[ps];
        for (int64_t j = 1; j < cnt; ++j) {
          int64_t dist = ecr[(size_t)(ps + j)] - col_start[(size_t)g];
          if (dist >= nL) {
            g++;
            col_start.push_back(ecr[(size_t)(ps + j)]);
            val_align.resize(val_align.size() + nL, T(0));
            dist = 0;
          }
          val_align[(size_t)(g * nL + dist)] = A.Val[ps + j];
        }
        g++;
      }
      v_row_ptr[(size_t)i + 1] = (int)g;
    }
  }
  // rows never visited (none in a valid partition) keep the running count
  for (int64_t i = 0; i < m; ++i) v_row_ptr[(size_t)i + 1] = std::max(v_row_ptr[(size_t)i + 1], v_row_ptr[(size_t)i]);
  const float ird = (g > 0) ? (float)nnz / (float)(g * nL) : 0.f;
  int64_t variant;
  if (force >= 0) variant = force;
  else if (m < 2000000) variant = (ird >= thr) ? 0 : 1;
  else variant = 2;
  auto* out = new Bundle();
  out->fmt = "vnec";
  out->set("m", (double)m); out->set("n", (double)n); out->set("nz", (double)nnz);
  out->set("NUM_THREADS_VNEC", (double)NT); out->set("nLanes", nL);
  out->set("IRD_mat", ird); out->set("vnec_t", (double)variant); out->set("dtype", dt_of<T>());
  out->put("ptr", ORC_I32, std::vector<int>(A.Rst, A.Rst + m + 1));
  out->put("indices", ORC_I32, std::vector<int>(A.Col, A.Col + nnz));
  out->put("val", dt_of<T>(), std::vector<T>(A.Val, A.Val + nnz));
  out->put("thread_coord_start", ORC_I32, tcs);
  out->put("thread_coord_end", ORC_I32, tce);
  if (variant == 0) {
    out->put("ecr_indices", ORC_I32, ecr);
    out->put("NEC_NUM", ORC_I32, nec);
    out->put("use_x_ptr", ORC_I32, ux_ptr);
    out->put("use_x_indices", ORC_I32, ux);
    out->put("v_row_ptr", ORC_I32, v_row_ptr);
    out->put("col_start", ORC_I32, col_start);
    out->put("val_align", dt_of<T>(), val_align);
  } else if (variant == 1) {
    // S: whole rows per thread, contiguous ranges balanced by nnz + rows
    std::vector<int> tstart((size_t)NT), tend((size_t)NT), spvv((size_t)NT), nec_s((size_t)NT);
    std::vector<int> uxs_ptr((size_t)NT + 1, 0), uxs, tasks, rbeg, rend, rcol;
    std::vector<T> rval;
    std::vector<int> row_lo((size_t)NT + 1);
    for (int64_t t = 0; t <= NT; ++t) {
      int64_t d = std::min(ipt * t, items), x, yv;
      merge_path(d, A.Rst + 1, m, nnz, &x, &yv);
      row_lo[(size_t)t] = (int)x;
    }
    row_lo[(size_t)NT] = (int)m;
    for (int64_t t = 0; t < NT; ++t) {
      int64_t r0 = row_lo[(size_t)t], r1 = std::max<int64_t>(r0, row_lo[(size_t)t + 1]);
      std::vector<int> used;
      for (int64_t r = r0; r < r1; ++r)
        for (int64_t k = A.Rst[r]; k < A.Rst[r + 1]; ++k)
          if (mark[(size_t)A.Col[k]] != (int)(NT + t)) { mark[(size_t)A.Col[k]] = (int)(NT + t); used.push_back(A.Col[k]); }
      std::sort(used.begin(), used.end());
      for (size_t k = 0; k < used.size(); ++k) rank[(size_t)used[k]] = (int)k;
      nec_s[(size_t)t] = (int)used.size();
      uxs.insert(uxs.end(), used.begin(), used.end());
      uxs_ptr[(size_t)t + 1] = (int)uxs.size();
      std::vector<int> shortr, longr;
      for (int64_t r = r0; r < r1; ++r) ((A.Rst[r + 1] - A.Rst[r]) < nL ? shortr : longr).push_back((int)r);
      std::stable_sort(shortr.begin(), shortr.end(), [&](int a, int b) {
        return (A.Rst[a + 1] - A.Rst[a]) > (A.Rst[b + 1] - A.Rst[b]);
      });
      int64_t ngroups = (int64_t)shortr.size() / nL;
      std::vector<int> inrow(shortr.begin() + ngroups * nL, shortr.end());
      inrow.insert(inrow.end(), longr.begin(), longr.end());
      tstart[(size_t)t] = (int)tasks.size();
      spvv[(size_t)t] = (int)(ngroups * nL);
      for (int64_t q = 0; q < ngroups; ++q) {
        int64_t rl = A.Rst[shortr[(size_t)(q * nL)] + 1] - A.Rst[shortr[(size_t)(q * nL)]];
        int base = (int)rcol.size();
        rcol.resize(rcol.size() + (size_t)(rl * nL), 0);
        rval.resize(rval.size() + (size_t)(rl * nL), T(0));
        for (int64_t k = 0; k < nL; ++k) {
          int r = shortr[(size_t)(q * nL + k)];
          tasks.push_back(r);
          rbeg.push_back(base);
          rend.push_back(base + (int)rl);
          for (int64_t c = 0; c < A.Rst[r + 1] - A.Rst[r]; ++c) {
            rcol[(size_t)(base + c * nL + k)] = rank[(size_t)A.Col[A.Rst[r] + c]];
            rval[(size_t)(base + c * nL + k)] = A.Val[A.Rst[r] + c];
          }
        }
      }
      for (int r : inrow) {
        tasks.push_back(r);
        rbeg.push_back((int)rcol.size());
        for (int64_t k = A.Rst[r]; k < A.Rst[r + 1]; ++k) { rcol.push_back(rank[(size_t)A.Col[k]]); rval.push_back(A.Val[k]); }
        rend.push_back((int)rcol.size());
      }
      tend[(size_t)t] = (int)tasks.size();
    }
    out->put("NEC_NUM", ORC_I32, nec_s);
    out->put("use_x_ptr", ORC_I32, uxs_ptr);
    out->put("use_x_indices", ORC_I32, uxs);
    out->put("tasks", ORC_I32, tasks);
    out->put("task_start", ORC_I32, tstart);
    out->put("task_end", ORC_I32, tend);
    out->put("spvv_len", ORC_I32, spvv);
    out->put("row_begin", ORC_I32, rbeg);
    out->put("row_end", ORC_I32, rend);
    out->put("reorder_col", ORC_I32, rcol);
    out->put("reorder_nnz", dt_of<T>(), rval);
  }
  return out;
}

template <class T>
void vnec_spmv(const Bundle& B, T alpha, const T* x, T beta, T* y) {
  const int64_t m = B.i("m"), NT = B.i("NUM_THREADS_VNEC"), nL = B.i("nLanes"), variant = B.i("vnec_t");
  const int* ptr = B.get<int>("ptr");
  const int* ind = B.get<int>("indices");
  const T* val = B.get<T>("val");
  const int* tcs = B.get<int>("thread_coord_start");
  const int* tce = B.get<int>("thread_coord_end");
  if (variant == 1) {  // S — spmv_mtx_vnec.cpp:199-282
    const int* ux_ptr = B.get<int>("use_x_ptr");
    const int* ux = B.get<int>("use_x_indices");
    const int* nec = B.get<int>("NEC_NUM");
    const int* tasks = B.get<int>("tasks");
    const int* ts = B.get<int>("task_start");
    const int* te = B.get<int>("task_end");
    const int* sv = B.get<int>("spvv_len");
    const int* rb = B.get<int>("row_begin");
    const int* re = B.get<int>("row_end");
    const int* rc = B.get<int>("reorder_col");
    const T* rv = B.get<T>("reorder_nnz");
    for (int64_t t = 0; t < NT; ++t) {
      std::vector<T> xx((size_t)nec[t] + (size_t)nL, T(0));
      for (int64_t j = 0; j < nec[t]; ++j) xx[(size_t)j] = x[ux[ux_ptr[t] + j]];
      const int* rows = tasks + ts[t];
      int64_t p = ts[t], c = 0;
      for (; c < sv[t]; p += nL, c += nL) {  // cross-row :89-101
        int64_t rl = re[p] - rb[p], base = rb[p];
        for (int64_t k = 0; k < nL; ++k) {
          T acc = 0;
          for (int64_t q = 0; q < rl; ++q) acc += rv[base + q * nL + k] * xx[(size_t)rc[base + q * nL + k]];
          int r = rows[c + k];
          T yy = y[r] * beta;
          y[r] = acc * alpha + yy;
        }
      }
      for (; p < te[t]; ++p) {  // in-row :103-133
        int r = rows[p - ts[t]];
        T s = 0;
        for (int64_t q = rb[p]; q < re[p]; ++q) s += rv[q] * xx[(size_t)rc[q]];
        y[r] = beta * y[r] + alpha * s;
      }
    }
    return;
  }
  for (int64_t i = 0; i < m; ++i) y[i] *= beta;  // D :289-307, L :465-482
  std::vector<int64_t> crow((size_t)NT);
  std::vector<T> cval((size_t)NT);
  for (int64_t t = 0; t < NT; ++t) {
    int64_t sx = tcs[2 * t], sy = tcs[2 * t + 1], ex = tce[2 * t], ey = tce[2 * t + 1];
    if (variant == 0) {  // D :309-353
      const int* ux_ptr = B.get<int>("use_x_ptr");
      const int* ux = B.get<int>("use_x_indices");
      const int* nec = B.get<int>("NEC_NUM");
      const int* ecr = B.get<int>("ecr_indices");
      const int* vrp = B.get<int>("v_row_ptr");
      const int* cs = B.get<int>("col_start");
      const T* va = B.get<T>("val_align");
      std::vector<T> xx((size_t)nec[t] + (size_t)nL, T(0));
      for (int64_t j = 0; j < nec[t]; ++j) xx[(size_t)j] = x[ux[ux_ptr[t] + j]];
      for (int64_t i = sx; i < ex; ++i) {
        std::vector<T> lane((size_t)nL, T(0));
        for (int64_t gg = vrp[i]; gg < vrp[i + 1]; ++gg)
          for (int64_t k = 0; k < nL; ++k) lane[(size_t)k] += va[gg * nL + k] * xx[(size_t)(cs[gg] + k)];
        T tmp = 0;
        for (int64_t k = 0; k < nL; ++k) tmp += lane[(size_t)k];
        y[i] = y[i] + alpha * tmp;
      }
      // carry: the thread's share of row ex (the reference starts at
      // ptr[ex] (:345), which re-reads the previous thread's share when the
      // thread completes no row; the share starts at max(ptr[ex], sy))
      T run = 0;
      int64_t k0 = (ex < m) ? std::max<int64_t>(ptr[ex], sy) : ey;
      for (int64_t k = k0; k < ey; ++k) run += val[k] * xx[(size_t)ecr[k]];
      crow[(size_t)t] = ex;
      cval[(size_t)t] = run;
    } else {  // L :484-520
      for (; sx < ex; ++sx) {
        T run = 0;
        for (; sy < ptr[sx + 1]; ++sy) run += val[sy] * x[ind[sy]];
        y[sx] += alpha * run;
      }
      T run = 0;
      for (; sy < ey; ++sy) run += val[sy] * x[ind[sy]];
      crow[(size_t)t] = ex;
      cval[(size_t)t] = run;
    }
  }
  for (int64_t t = 0; t + 1 < NT; ++t)  // carry fix-up :355-359, :522-526
    if (crow[(size_t)t] < m) y[crow[(size_t)t]] += alpha * cval[(size_t)t];
}

// =====================================================================
// VHCC builder (include/VHCC.h:80-112 has setters for a builder that is
// missing).  One panel.  Layout as read by vhcc_spmv_1panel_riscv
// (src/rvv/spmv_vhcc.cpp:73-162 fp64, :164-250 fp32):
//   nonzeros in CSR order packed into vectors of vec_size lanes (zero padded);
//   threads own equal vector ranges [start_vec, end_vec);
//   a "write lane" ends a row (its last nonzero) or ends a thread range (the
//   thread's last lane, written to the thread's overflow row num_rows+tid
//   unless a row ends there);
//   veceor_ptr lists, per thread in order, the vectors holding a write lane,
//   then one sentinel (num_vectors);
//   per such vector: n_masks scan masks (offset 1,2,4..: bit i set when i >= d
//   and lanes i-d..i-1 hold no write lane) then the write mask, each
//   vec_size/8 bytes; row_arr lists the write lanes' rows in order;
//   thr_info: vbase/rbase index veceor_ptr/row_arr, sbase = vbase *
//   (n_masks+1) * vec_size/8 (bytes); last_row += tmp[overflow_row] after the
//   barrier (:157-161).
// =====================================================================
template <class T>
Bundle* build_vhcc(const Crs<T>& A, int64_t NT, int64_t vec) {
  if (NT <= 0) throw std::invalid_argument("VHCC: num_threads must be positive");
  if (vec < 8 || (vec & (vec - 1))) throw std::invalid_argument("VHCC: vec_size must be a power of two >= 8");
  const int64_t m = A.m, nnz = A.nz;
  const int nm = bits_for(vec) - 1;
  const int64_t mb = vec / 8;
  const int64_t nvec = (nnz + vec - 1) / vec;
  std::vector<int> rowof((size_t)(nvec * vec), -1);
  for (int64_t r = 0; r < m; ++r)
    for (int64_t k = A.Rst[r]; k < A.Rst[r + 1]; ++k) rowof[(size_t)k] = (int)r;
  std::vector<uint8_t> is_end((size_t)(nvec * vec), 0);
  for (int64_t r = 0; r < m; ++r)
    if (A.Rst[r + 1] > A.Rst[r]) is_end[(size_t)(A.Rst[r + 1] - 1)] = 1;
  std::vector<uint32_t> col((size_t)(nvec * vec), 0u), rows_arr, veceor;
  std::vector<T> vals((size_t)(nvec * vec), T(0));
  for (int64_t k = 0; k < nnz; ++k) { col[(size_t)k] = (uint32_t)A.Col[k]; vals[(size_t)k] = A.Val[k]; }
  std::vector<uint8_t> smask;
  std::vector<int> thr((size_t)NT * 10, 0);
  for (int64_t t = 0; t < NT; ++t) {
    int64_t v0 = nvec * t / NT, v1 = nvec * (t + 1) / NT;
    int* ti = thr.data() + t * 10;
    ti[0] = (int)veceor.size();           // vbase
    ti[1] = (int)rows_arr.size();         // rbase
    ti[2] = (int)(veceor.size() * (size_t)(nm + 1) * (size_t)mb);  // sbase (bytes)
    ti[3] = (int)(m + t);                 // last_row (patched below)
    ti[4] = (int)(m + t);                 // overflow_row
    ti[5] = (int)v0; ti[6] = (int)v1;     // start_vec, end_vec
    ti[7] = 0; ti[8] = 0; ti[9] = 0;      // panel_id, merge_start, merge_end
    for (int64_t v = v0; v < v1; ++v) {
      std::vector<uint8_t> w((size_t)vec, 0);
      for (int64_t l = 0; l < vec; ++l) w[(size_t)l] = is_end[(size_t)(v * vec + l)];
      bool thread_end = (v == v1 - 1);
      bool real_end_last = w[(size_t)(vec - 1)] != 0;
      if (thread_end) w[(size_t)(vec - 1)] = 1;
      bool any = false;
      for (auto b : w) any |= (b != 0);
      if (!any) continue;
      veceor.push_back((uint32_t)v);
      for (int sidx = 0; sidx < nm; ++sidx) {
        int64_t d = int64_t(1) << sidx;
        std::vector<uint8_t> bytes((size_t)mb, 0);
        for (int64_t i = d; i < vec; ++i) {
          bool ok = true;
          for (int64_t q = i - d; q < i; ++q) ok &= !w[(size_t)q];
          if (ok) bytes[(size_t)(i / 8)] |= (uint8_t)(1u << (i % 8));
        }
        smask.insert(smask.end(), bytes.begin(), bytes.end());
      }
      std::vector<uint8_t> wb((size_t)mb, 0);
      for (int64_t i = 0; i < vec; ++i)
        if (w[(size_t)i]) wb[(size_t)(i / 8)] |= (uint8_t)(1u << (i % 8));
      smask.insert(smask.end(), wb.begin(), wb.end());
      for (int64_t l = 0; l < vec; ++l) {
        if (!w[(size_t)l]) continue;
        if (thread_end && l == vec - 1 && !real_end_last) {
          rows_arr.push_back((uint32_t)(m + t));
          // the interrupted row (or, past the last nonzero, the last row)
          int64_t k = v * vec + l;
          int r = (k < nnz) ? rowof[(size_t)k] : (nnz > 0 ? rowof[(size_t)(nnz - 1)] : 0);
          ti[3] = r;
        } else {
          rows_arr.push_back((uint32_t)rowof[(size_t)(v * vec + l)]);
        }
      }
    }
  }
  veceor.push_back((uint32_t)nvec);  // sentinel read after a thread's last EOR vector
  auto* out = new Bundle();
  out->fmt = "vhcc";
  out->set("num_rows", (double)m); out->set("num_cols", (double)A.n);
  out->set("num_entries", (double)nnz); out->set("num_vectors", (double)nvec);
  out->set("pad_entries", (double)(nvec * vec - nnz)); out->set("pad_rows", (double)(m + NT));
  out->set("num_threads", (double)NT); out->set("num_panels", 1);
  out->set("tile_row", 512); out->set("tile_col", 512);
  out->set("vec_size", (double)vec); out->set("n_masks", nm); out->set("dtype", dt_of<T>());
  out->put("thr_info", ORC_I32, thr);
  out->put("veceor_ptr", ORC_U32, veceor);
  out->put("scan_mask", ORC_U8, smask);
  out->put("row_arr", ORC_U32, rows_arr);
  out->put("col_arr", ORC_U32, col);
  out->put("vals_arr", dt_of<T>(), vals);
  return out;
}

// VHCC SpMV — restates vhcc_spmv_1panel_riscv (src/rvv/spmv_vhcc.cpp:73-162)
// for any vec_size, then the alpha/beta epilogue of :335-397.
template <class T>
void vhcc_spmv(const Bundle& B, T alpha, const T* x, T beta, T* y) {
  const int64_t m = B.i("num_rows"), NT = B.i("num_threads"), vec = B.i("vec_size"), nm = B.i("n_masks");
  const int64_t mb = vec / 8, pad_rows = B.i("pad_rows");
  const int* thr = B.get<int>("thr_info");
  const uint32_t* veceor = B.get<uint32_t>("veceor_ptr");
  const uint8_t* smask = B.get<uint8_t>("scan_mask");
  const uint32_t* rows = B.get<uint32_t>("row_arr");
  const uint32_t* col = B.get<uint32_t>("col_arr");
  const T* vals = B.get<T>("vals_arr");
  std::vector<T> tmp((size_t)pad_rows, T(0));
  auto bit = [&](const uint8_t* mk, int64_t i) { return (mk[i / 8] >> (i % 8)) & 1; };
  for (int64_t t = 0; t < NT; ++t) {
    const int* ti = thr + t * 10;
    int64_t vidx = ti[0], sidx = (int64_t)ti[2], ridx = ti[1];
    uint32_t eor = veceor[vidx++];
    std::vector<T> res((size_t)vec, T(0));
    for (int64_t v = ti[5]; v < ti[6]; ++v) {
      for (int64_t l = 0; l < vec; ++l) res[(size_t)l] += vals[v * vec + l] * x[col[v * vec + l]];
      if ((uint32_t)v == eor) {
        for (int64_t s = 0; s < nm; ++s) {  // masked slide-up scan :113-120
          int64_t d = int64_t(1) << s;
          const uint8_t* mk = smask + sidx;
          std::vector<T> prev = res;
          for (int64_t l = d; l < vec; ++l)
            if (bit(mk, l)) res[(size_t)l] = prev[(size_t)l] + prev[(size_t)(l - d)];
          sidx += mb;
        }
        const uint8_t* wm = smask + sidx;
        sidx += mb;
        for (int64_t l = 0; l < vec; ++l)  // compress + scatter :30-46
          if (bit(wm, l)) { tmp[rows[ridx]] += res[(size_t)l]; ridx++; }
        eor = veceor[vidx++];
        T carry = bit(wm, vec - 1) ? T(0) : res[(size_t)(vec - 1)];
        std::fill(res.begin(), res.end(), T(0));
        res[0] = carry;
      } else {
        T s = 0;
        for (int64_t l = 0; l < vec; ++l) s += res[(size_t)l];
        std::fill(res.begin(), res.end(), T(0));
        res[0] = s;
      }
    }
  }
  for (int64_t t = 0; t < NT; ++t) {  // :157-161
    const int* ti = thr + t * 10;
    tmp[(size_t)ti[3]] += tmp[(size_t)ti[4]];
  }
  for (int64_t i = 0; i < m; ++i) y[i] = beta * y[i] + alpha * tmp[(size_t)i];
}

// =====================================================================
// CVR builder (no reference builder).  Layout as read by
// src/scalar/spmv_mtx_cvr.cpp:32-66:
//   vPack_vec_vals/cols: SIMD_LEN lanes per vector; a lane streams the
//   nonzeros of one row after another;
//   vPack_vec_record: pairs (pos, row), sorted by pos: before accumulating the
//   vector holding pos, lane pos % SIMD_LEN is flushed into y[row] (so pos is
//   the lane's first slot after row ends), plus a trailing ignored pair;
//   writeback_pos_record: Nthreads blocks of SIMD_LEN+2 ints: [first vector,
//   first record pair, tail row of each lane]; the kernel flushes the last
//   block's tail rows after the final vector.
// Threads own contiguous whole-row ranges balanced by nonzeros; inside a
// range, rows enter lanes longest first (stable), empty rows are skipped;
// every lane still holding a row at a range end (except the last range) gets
// a record at the next range's first vector.
// =====================================================================
template <class T>
Bundle* build_cvr(const Crs<T>& A, int64_t S, int64_t NT) {
  if (S <= 0 || NT <= 0) throw std::invalid_argument("CVR: SIMD_LEN and Nthreads must be positive");
  const int64_t m = A.m, nnz = A.nz;
  std::vector<T> vals;
  std::vector<uint32_t> cols;
  std::vector<int> rec, wb((size_t)(NT * (S + 2)), 0);
  std::vector<int64_t> bounds((size_t)NT + 1, m);
  bounds[0] = 0;
  for (int64_t t = 1; t < NT; ++t) {
    int64_t target = nnz * t / NT;
    bounds[(size_t)t] = std::upper_bound(A.Rst, A.Rst + m + 1, (int)target) - A.Rst - 1;
    bounds[(size_t)t] = std::max(bounds[(size_t)t], bounds[(size_t)t - 1]);
  }
  int64_t nv = 0;
  for (int64_t t = 0; t < NT; ++t) {
    int* blk = wb.data() + t * (S + 2);
    blk[0] = (int)nv;
    blk[1] = (int)(rec.size() / 2);
    std::vector<int> rows;
    for (int64_t r = bounds[(size_t)t]; r < bounds[(size_t)t + 1]; ++r)
      if (A.Rst[r + 1] > A.Rst[r]) rows.push_back((int)r);
    std::stable_sort(rows.begin(), rows.end(), [&](int a, int b) {
      return (A.Rst[a + 1] - A.Rst[a]) > (A.Rst[b + 1] - A.Rst[b]);
    });
    size_t next = 0;
    std::vector<int> lrow((size_t)S, -1);
    std::vector<int64_t> lpos((size_t)S, 0), lend((size_t)S, 0);
    for (;;) {
      bool any = false;
      for (int64_t l = 0; l < S; ++l) {
        if (lrow[(size_t)l] >= 0 && lpos[(size_t)l] == lend[(size_t)l]) {
          rec.push_back((int)(nv * S + l));
          rec.push_back(lrow[(size_t)l]);
          lrow[(size_t)l] = -1;
        }
        if (lrow[(size_t)l] < 0 && next < rows.size()) {
          int r = rows[next++];
          lrow[(size_t)l] = r;
          lpos[(size_t)l] = A.Rst[r];
          lend[(size_t)l] = A.Rst[r + 1];
        }
        any |= lrow[(size_t)l] >= 0;
      }
      if (!any) break;
      for (int64_t l = 0; l < S; ++l) {
        if (lrow[(size_t)l] >= 0 && lpos[(size_t)l] < lend[(size_t)l]) {
          vals.push_back(A.Val[lpos[(size_t)l]]);
          cols.push_back((uint32_t)A.Col[lpos[(size_t)l]]);
          lpos[(size_t)l]++;
        } else {
          vals.push_back(T(0));
          cols.push_back(0u);
        }
      }
      nv++;
      // drop lanes whose row is finished and nothing is left to schedule,
      // unless they must be flushed: their record is emitted at the next
      // vector above, or by the range-end pass below
      bool more = next < rows.size();
      if (!more) {
        bool pending = false;
        for (int64_t l = 0; l < S; ++l) pending |= (lrow[(size_t)l] >= 0 && lpos[(size_t)l] < lend[(size_t)l]);
        if (!pending) break;
      }
    }
    for (int64_t l = 0; l < S; ++l) {
      int r = lrow[(size_t)l];
      if (t + 1 < NT) {
        if (r >= 0) { rec.push_back((int)(nv * S + l)); rec.push_back(r); }
        blk[2 + l] = 0;
      } else {
        blk[2 + l] = r >= 0 ? r : 0;
      }
    }
  }
  rec.push_back((int)(nv * S));
  rec.push_back(0);
  auto* out = new Bundle();
  out->fmt = "cvr";
  out->set("nItems", (double)(nv * S)); out->set("numRows", (double)m); out->set("numCols", (double)A.n);
  out->set("SIMD_LEN", (double)S); out->set("Nthreads", (double)NT); out->set("Nthreads_avail", (double)NT);
  out->set("dtype", dt_of<T>());
  out->put("vPack_vec_vals", dt_of<T>(), vals);
  out->put("vPack_vec_cols", ORC_U32, cols);
  out->put("vPack_vec_record", ORC_I32, rec);
  out->put("writeback_pos_record", ORC_I32, wb);
  return out;
}

// CVR SpMV — src/scalar/spmv_mtx_cvr.cpp:21-68, restated.
template <class T>
void cvr_spmv(const Bundle& B, T alpha, const T* b, T beta, T* y) {
  const int64_t nItems = B.i("nItems"), m = B.i("numRows"), S = B.i("SIMD_LEN"), NTa = B.i("Nthreads_avail");
  int64_t nrec;
  const T* vals = B.get<T>("vPack_vec_vals");
  const uint32_t* cols = B.get<uint32_t>("vPack_vec_cols");
  const int* rec = B.get<int>("vPack_vec_record", &nrec);
  const int* wb = B.get<int>("writeback_pos_record");
  for (int64_t i = 0; i < m; ++i) y[i] *= beta;
  std::vector<T> res((size_t)S, T(0));
  int64_t ir = 0, irmax = (nrec - 2) / 2, lb = 0;
  while (ir < irmax) {
    for (; lb + S <= rec[2 * ir]; lb += S)
      for (int64_t i = 0; i < S; ++i) res[(size_t)i] += vals[lb + i] * b[cols[lb + i]];
    int64_t pos = rec[2 * ir] % S;
    y[rec[2 * ir + 1]] += alpha * res[(size_t)pos];
    res[(size_t)pos] = 0;
    ir++;
  }
  for (; lb + S <= nItems; lb += S)
    for (int64_t i = 0; i < S; ++i) res[(size_t)i] += vals[lb + i] * b[cols[lb + i]];
  if (m > 0) {
    const int* tail = wb + (NTa - 1) * (S + 2) + 2;
    for (int64_t i = 0; i < S; ++i) y[tail[i]] += alpha * res[(size_t)i];
  }
}

// ---------------------------------------------------------------- format -> CSR
template <class T>
Bundle* to_crs(const Bundle& B) {
  // Reconstruct (row, col, val) triples from the format, then sort by (row,
  // position in row as stored).  Used by the round-trip tests.
  std::vector<std::vector<std::pair<int, T>>> rows;
  int64_t m = 0, n = 0;
  const std::string& f = B.fmt;
  if (f == "crs") {
    Crs<T> A = crs_view<T>(B);
    return new_crs<T>(A.m, A.n, std::vector<int>(A.Rst, A.Rst + A.m + 1), std::vector<int>(A.Col, A.Col + A.nz),
                      std::vector<T>(A.Val, A.Val + A.nz));
  } else if (f == "hcsr") {
    m = B.i("m"); n = B.i("n");
    rows.resize((size_t)m);
    const int64_t R = B.i("R"), C = B.i("C"), b_m = B.i("b_m"), b_n = B.i("b_n");
    const int* bp = B.get<int>("block_ptr");
    const uint32_t* ro = B.get<uint32_t>("row_offset");
    const uint32_t* rp = B.get<uint32_t>("row_ptr");
    const uint16_t* ci = B.get<uint16_t>("col_idx");
    const T* v = B.get<T>("values");
    for (int64_t br = 0; br < b_m; ++br)
      for (int64_t bc = 0; bc < b_n; ++bc) {
        int64_t blk = br * b_n + bc;
        uint32_t key = ro[blk] >> 30, off = ro[blk] & 0x3FFFFFFFu;
        int64_t maxr = std::min(R, m - br * R);
        if (key == 1) {
          for (int64_t r = 0; r < maxr; ++r)
            for (uint32_t q = rp[off + r]; q < rp[off + r + 1]; ++q)
              rows[(size_t)(br * R + r)].emplace_back((int)(bc * C + ci[bp[blk] + q]), v[bp[blk] + q]);
        } else {
          for (int64_t q = 0; q < bp[blk + 1] - bp[blk]; ++q)
            rows[(size_t)(br * R + rp[off + q])].emplace_back((int)(bc * C + ci[bp[blk] + q]), v[bp[blk] + q]);
        }
      }
  } else if (f == "sell") {
    m = B.i("m"); n = B.i("n");
    rows.resize((size_t)m);
    const int64_t cnt_b = B.i("cnt_b");
    const int* Cl = B.get<int>("vCl");
    const int* Cs = B.get<int>("vCs");
    const int* Bs = B.get<int>("vBs");
    const int* SBs = B.get<int>("vSBs");
    const uint32_t* Col = B.get<uint32_t>("vCol");
    const uint32_t* Perm = B.get<uint32_t>("vPerm");
    const T* Val = B.get<T>("vVal");
    for (int64_t s = 0; s < cnt_b; ++s)
      for (int64_t k = 0; k < Bs[s]; ++k)
        for (int64_t j = 0; j < Cl[s]; ++j) {
          int64_t q = Cs[s] + j * Bs[s] + k;
          if (Val[q] != T(0)) rows[Perm[SBs[s] + k]].emplace_back((int)Col[q], Val[q]);
        }
  } else if (f == "csr5") {
    m = B.i("m"); n = B.i("n");
    rows.resize((size_t)m);
    const int64_t p = B.i("p"), w = B.i("omega"), s = B.i("sigma"), nnz = B.i("nnz");
    const int* rp = B.get<int>("csr_row_pointer");
    const uint32_t* ci = B.get<uint32_t>("csr_column_index");
    const T* cv = B.get<T>("csr_value");
    for (int64_t r = 0; r < m; ++r)
      for (int64_t k = rp[r]; k < rp[r + 1]; ++k) {
        int64_t t = k / (w * s), q = k;
        if (t < p - 1) { int64_t e = k - t * w * s; q = t * w * s + (e % s) * w + e / s; }
        (void)nnz;
        rows[(size_t)r].emplace_back((int)ci[q], cv[q]);
      }
  } else {
    throw std::runtime_error("to_crs: unsupported format " + f);
  }
  std::vector<int> Rst((size_t)m + 1, 0), Col;
  std::vector<T> Val;
  for (int64_t r = 0; r < m; ++r) {
    auto& e = rows[(size_t)r];
    std::stable_sort(e.begin(), e.end(), [](const std::pair<int, T>& a, const std::pair<int, T>& b) { return a.first < b.first; });
    for (auto& pr : e) { Col.push_back(pr.first); Val.push_back(pr.second); }
    Rst[(size_t)r + 1] = (int)Col.size();
  }
  return new_crs<T>(m, n, Rst, Col, Val);
}

template <class T>
Bundle* transpose(const Crs<T>& A) {
  std::vector<int> Rt((size_t)A.n + 1, 0), Ct((size_t)A.nz), perm((size_t)A.nz);
  std::vector<T> Vt((size_t)A.nz);
  for (int64_t k = 0; k < A.nz; ++k) Rt[(size_t)A.Col[k] + 1]++;
  for (int64_t c = 0; c < A.n; ++c) Rt[(size_t)c + 1] += Rt[(size_t)c];
  std::vector<int> nx(Rt.begin(), Rt.end() - 1);
  for (int64_t r = 0; r < A.m; ++r)
    for (int64_t k = A.Rst[r]; k < A.Rst[r + 1]; ++k) {
      int q = nx[(size_t)A.Col[k]]++;
      Ct[(size_t)q] = (int)r;
      Vt[(size_t)q] = A.Val[k];
      perm[(size_t)q] = (int)k;
    }
  Bundle* b = new_crs<T>(A.n, A.m, Rt, Ct, Vt);
  b->put("perm", ORC_I32, perm);
  return b;
}

template <class F>
void* guarded(F&& f) {
  try {
    return f();
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

template <template <class> class Fn, class... Args>
void* by_dtype(void* crs, Args... args) {
  return guarded([&]() -> void* {
    const Bundle& b = *(Bundle*)crs;
    if (val_dtype(b) == ORC_F32) return Fn<float>::run(crs_view<float>(b), args...);
    return Fn<double>::run(crs_view<double>(b), args...);
  });
}

template <class T> struct HcsrB { static Bundle* run(const Crs<T>& A, int64_t R, int64_t C, double p) { return build_hcsr(A, R, C, p); } };
template <class T> struct SellB { static Bundle* run(const Crs<T>& A, int64_t C, int64_t s) { return build_sell(A, C, s); } };
template <class T> struct Csr5B { static Bundle* run(const Crs<T>& A, int64_t w, int64_t s) { return build_csr5(A, w, s); } };
template <class T> struct LavB { static Bundle* run(const Crs<T>& A, int64_t L, double Tt, int64_t sl) { return build_lav(A, L, Tt, sl); } };
template <class T> struct VnecB { static Bundle* run(const Crs<T>& A, int64_t nt, int64_t f) { return build_vnec(A, nt, f); } };
template <class T> struct VhccB { static Bundle* run(const Crs<T>& A, int64_t nt, int64_t v) { return build_vhcc(A, nt, v); } };
template <class T> struct CvrB { static Bundle* run(const Crs<T>& A, int64_t s, int64_t nt) { return build_cvr(A, s, nt); } };
template <class T> struct TrB { static Bundle* run(const Crs<T>& A) { return transpose(A); } };

template <class T>
int spmv_t(const Bundle& B, double alpha, const void* b, double beta, void* y, int stage) {
  const T a = (T)alpha, be = (T)beta;
  const T* bb = (const T*)b;
  T* yy = (T*)y;
  const std::string& f = B.fmt;
  if (f == "crs") crs_spmv(crs_view<T>(B), a, bb, be, yy);
  else if (f == "hcsr") hcsr_spmv(B, a, bb, be, yy);
  else if (f == "sell") sell_spmv(B, a, bb, be, yy, stage);
  else if (f == "csr5") csr5_spmv(B, a, bb, be, yy);
  else if (f == "lav") lav_spmv(B, a, bb, be, yy);
  else if (f == "vnec") vnec_spmv(B, a, bb, be, yy);
  else if (f == "vhcc") vhcc_spmv(B, a, bb, be, yy);
  else if (f == "cvr") cvr_spmv(B, a, bb, be, yy);
  else { g_err = "spmv: unknown format " + f; return -1; }
  return 0;
}

}  // namespace

extern "C" {

void* orc_bundle_new(const char* fmt) { auto* b = new Bundle(); b->fmt = fmt; return b; }
void orc_bundle_free(void* h) { delete (Bundle*)h; }
const char* orc_bundle_fmt(void* h) { return ((Bundle*)h)->fmt.c_str(); }
void orc_bundle_put(void* h, const char* name, int dtype, const void* data, int64_t len) {
  Bundle* b = (Bundle*)h;
  Arr a;
  a.name = name;
  a.dtype = dtype;
  a.len = len;
  a.bytes.resize((size_t)(len * dtype_size(dtype)));
  if (len > 0) std::memcpy(a.bytes.data(), data, a.bytes.size());
  for (auto& e : b->arrs)
    if (e.name == a.name) { e = std::move(a); return; }
  b->arrs.push_back(std::move(a));
}
int orc_bundle_count(void* h) { return (int)((Bundle*)h)->arrs.size(); }
const char* orc_bundle_name(void* h, int i) { return ((Bundle*)h)->arrs[(size_t)i].name.c_str(); }
int orc_bundle_dtype(void* h, int i) { return ((Bundle*)h)->arrs[(size_t)i].dtype; }
int64_t orc_bundle_len(void* h, int i) { return ((Bundle*)h)->arrs[(size_t)i].len; }
const void* orc_bundle_data(void* h, int i) { return ((Bundle*)h)->arrs[(size_t)i].bytes.data(); }
void orc_bundle_set(void* h, const char* name, double v) { ((Bundle*)h)->set(name, v); }
int orc_bundle_nscalars(void* h) { return (int)((Bundle*)h)->sc.size(); }
const char* orc_bundle_scalar_name(void* h, int i) { return ((Bundle*)h)->sc[(size_t)i].first.c_str(); }
double orc_bundle_scalar(void* h, int i) { return ((Bundle*)h)->sc[(size_t)i].second; }
const char* orc_last_error(void) { return g_err.c_str(); }

void* orc_build_hcsr(void* crs, int64_t R, int64_t C, double p) { return by_dtype<HcsrB>(crs, R, C, p); }
void* orc_build_sell(void* crs, int64_t C, int64_t sigma) { return by_dtype<SellB>(crs, C, sigma); }
void* orc_build_csr5(void* crs, int64_t omega, int64_t sigma) { return by_dtype<Csr5B>(crs, omega, sigma); }
void* orc_build_lav(void* crs, int64_t L, double T, int64_t seglen) { return by_dtype<LavB>(crs, L, T, seglen); }
void* orc_build_vnec(void* crs, int64_t nt, int64_t force) { return by_dtype<VnecB>(crs, nt, force); }
void* orc_build_vhcc(void* crs, int64_t nt, int64_t vec) { return by_dtype<VhccB>(crs, nt, vec); }
void* orc_build_cvr(void* crs, int64_t s, int64_t nt) { return by_dtype<CvrB>(crs, s, nt); }
void* orc_transpose(void* crs) { return by_dtype<TrB>(crs); }

void* orc_to_crs(void* fmt) {
  return guarded([&]() -> void* {
    const Bundle& b = *(Bundle*)fmt;
    if (val_dtype(b) == ORC_F32) return to_crs<float>(b);
    return to_crs<double>(b);
  });
}

int orc_spmv(void* fmt, double alpha, const void* b, double beta, void* y, int stage) {
  try {
    const Bundle& B = *(Bundle*)fmt;
    if (val_dtype(B) == ORC_F32) return spmv_t<float>(B, alpha, b, beta, y, stage);
    return spmv_t<double>(B, alpha, b, beta, y, stage);
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

void orc_crs_spmv_ld(void* crs, double alpha, const double* b, double beta, double* y) {
  Crs<double> A = crs_view<double>(*(Bundle*)crs);
  for (int64_t i = 0; i < A.m; ++i) {
    long double acc = 0;
    for (int64_t k = A.Rst[i]; k < A.Rst[i + 1]; ++k) acc += (long double)A.Val[k] * (long double)b[A.Col[k]];
    y[i] = (double)((long double)alpha * acc + (long double)beta * (long double)y[i]);
  }
}

void orc_sddmm(void* crs, const double* g, const double* x, double* dvals) {
  const Bundle& B = *(Bundle*)crs;
  const int64_t m = B.i("m");
  const int* Rst = B.get<int>("Rst");
  const int* Col = B.get<int>("Col");
  for (int64_t i = 0; i < m; ++i)
    for (int64_t k = Rst[i]; k < Rst[i + 1]; ++k) dvals[k] = g[i] * x[Col[k]];
}

void orc_merge_path(int64_t diagonal, const int* a, int64_t a_len, int64_t b_len, int64_t* out_xy) {
  merge_path(diagonal, a, a_len, b_len, &out_xy[0], &out_xy[1]);
}

}  // extern "C"
