// crs_run.cuh — CSR SpMV with lane-contiguous runs (the CSR5 idea applied to
// plain CSR storage, with a row-start bitmap from the analysis instead of
// CSR5's tile descriptors).
//
// Each warp owns a contiguous range of E nonzeros (the same ranges and first
// rows as the stream kernel).  A chunk is 256 nonzeros: lane l owns the 8
// consecutive nonzeros [c0 + 8l, c0 + 8l + 8), loaded with 128-bit loads
// through L1 (columns as two int4, values as 64 / 32 / 16 bytes), and bit k
// of the bitmap marks nonzero k as the first of its row.  Per lane, the 8 products
// are summed in order, splitting at the marked positions: rows that start and
// end inside the lane are written directly; the part before the lane's first
// mark (its "lead") belongs to the row open at the lane's start, the part
// after its last mark (its "tail") to the row open at its end.  A reverse
// segmented warp scan of the leads closes the rows that cross lanes, and the
// row open at the chunk end is carried in registers to the next chunk.  Row
// numbers come from a warp prefix sum of the marks.  Rows that cross a warp
// boundary leave (row, partial) carries added in warp order by the stream
// kernel's fix-up.  All sums run in a fixed order (bitwise reproducible).
#pragma once
#include "crs_merge.cuh"

namespace rvvla {

constexpr int kRunLane = 8;                 // nonzeros per lane in a chunk (16 measured slower)
constexpr int kRunChunk = 32 * kRunLane;    // nonzeros per chunk

// 16-byte loads through L1 (a warp's 16-byte pieces are 64 or 32 bytes
// apart, so the rest of each 32-byte sector is read by the next load) with
// the L2 evict-first hint.
__device__ __forceinline__ int4 ld_v4_l1(const void* p, uint64_t pol) {
  int4 v;
  asm("ld.global.nc.L2::cache_hint.v4.b32 {%0,%1,%2,%3}, [%4], %5;"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p), "l"(pol));
  return v;
}

template <class V> struct RunVec;
template <> struct RunVec<double> {
  __device__ static void load(const double* p, double (&v)[kRunLane], uint64_t pol) {
#pragma unroll
    for (int q = 0; q < kRunLane / 2; ++q) {
      const int4 t = ld_v4_l1(p + 2 * q, pol);
      v[2 * q] = __hiloint2double(t.y, t.x);
      v[2 * q + 1] = __hiloint2double(t.w, t.z);
    }
  }
};
template <> struct RunVec<float> {
  __device__ static void load(const float* p, float (&v)[kRunLane], uint64_t pol) {
#pragma unroll
    for (int q = 0; q < kRunLane / 4; ++q) {
      const int4 t = ld_v4_l1(p + 4 * q, pol);
      v[4 * q] = __int_as_float(t.x);
      v[4 * q + 1] = __int_as_float(t.y);
      v[4 * q + 2] = __int_as_float(t.z);
      v[4 * q + 3] = __int_as_float(t.w);
    }
  }
};
template <> struct RunVec<__nv_bfloat16> {
  __device__ static void load(const __nv_bfloat16* p, __nv_bfloat16 (&v)[kRunLane], uint64_t pol) {
#pragma unroll
    for (int q8 = 0; q8 < kRunLane / 8; ++q8) {
      const int4 t = ld_v4_l1(p + 8 * q8, pol);
      const unsigned w[4] = {(unsigned)t.x, (unsigned)t.y, (unsigned)t.z, (unsigned)t.w};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        v[8 * q8 + 2 * q] = __ushort_as_bfloat16((unsigned short)(w[q] & 0xFFFFu));
        v[8 * q8 + 2 * q + 1] = __ushort_as_bfloat16((unsigned short)(w[q] >> 16));
      }
    }
  }
};

// kRunLane 32-bit indices of a lane with 16-byte loads
__device__ __forceinline__ void run_idx(const int* p, int (&v)[kRunLane], uint64_t pol) {
#pragma unroll
  for (int q = 0; q < kRunLane / 4; ++q) {
    const int4 t = ld_v4_l1(p + 4 * q, pol);
    v[4 * q] = t.x;
    v[4 * q + 1] = t.y;
    v[4 * q + 2] = t.z;
    v[4 * q + 3] = t.w;
  }
}

// rst: row starts of the rows the warps walk (all rows, or the compacted
// non-empty rows with row_map back to the ids); bits: the row-start bitmap
// over the nonzeros; VEC: Col and Val (or perm) are 16-byte aligned (vector
// loads); PERM: value k is Val[perm[k]] (the adjoint reads A's values
// through the transpose's permutation instead of a re-gathered copy); DOT:
// every row piece v that leaves the kernel (stored, or handed on as a carry)
// also adds x[row] * v to the warp's partial dot_part[w], so the warps'
// partials sum to x^T (A x) without a second pass over y (the solvers'
// fused SpMV-dot; square A).
template <class V, class X, class Ac, class CT, bool VEC, bool PERM = false, bool DOT = false>
__global__ void __launch_bounds__(256)
crs_run_kernel(int m, int nnz, int E, int nwarps, const int* __restrict__ rst, const uint32_t* __restrict__ bits,
               const int* __restrict__ Col, const V* __restrict__ Val, const X* __restrict__ x, X* __restrict__ y,
               X alpha, X beta, const int* __restrict__ wrow, int* __restrict__ carry_row, CT* __restrict__ carry_val,
               const int* __restrict__ row_map, const int* __restrict__ perm = nullptr,
               CT* __restrict__ dot_part = nullptr) {
  const int w = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= nwarps) return;
  const int kb = w * E;
  const int ke = min(nnz, kb + E);
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  int crow = wrow[w];                     // the open row: row of the next nonzero
  const bool first_open = rst[crow] < kb;  // the warp's first row began in an earlier warp
  bool c_is_first = true;                  // the open row is the warp's first row
  CT cval = CT(0);
  int carry0_row = -1;
  CT carry0 = CT(0);
  auto yrow = [&](int r) { return row_map ? row_map[r] : r; };
  CT dotv = CT(0);  // DOT: this lane's share of x^T (A x)
  auto dot_add = [&](int r, CT v) {
    if constexpr (DOT) dotv += (CT)x[yrow(r)] * v;
  };
  // closes the open row (complete): the warp's first row may have begun in
  // an earlier warp, then it becomes a carry instead of a store
  auto close_open = [&](CT v) {
    if (lane == 0) dot_add(crow, v);
    if (c_is_first && first_open) {
      carry0_row = crow;
      carry0 = v;
    } else if (lane == 0) {
      write_row(y, yrow(crow), alpha, beta, (X)v);
    }
  };
  for (int c0 = kb; c0 < ke; c0 += kRunChunk) {
    const int a = c0 + kRunLane * lane;
    const int nv = max(0, min(kRunLane, ke - a));
    int cidx[kRunLane];
    V vv[kRunLane];
    if (VEC && c0 + kRunChunk <= ke) {
      run_idx(Col + a, cidx, pf);
      if constexpr (PERM) {
        int pi[kRunLane];
        run_idx(perm + a, pi, pf);
#pragma unroll
        for (int i = 0; i < kRunLane; ++i) vv[i] = Val[pi[i]];
      } else {
        RunVec<V>::load(Val + a, vv, pf);
      }
    } else {
#pragma unroll
      for (int i = 0; i < kRunLane; ++i) {
        const int k = i < nv ? a + i : kb;  // idle slots read a valid nonzero
        cidx[i] = ld_stream(Col + k, pf);
        if constexpr (PERM) vv[i] = Val[ld_stream(perm + k, pf)];
        else vv[i] = ld_stream(Val + k, pf);
      }
    }
    using PT = decltype(vmul(V(), X()));
    PT p[kRunLane];
#pragma unroll
    for (int i = 0; i < kRunLane; ++i) p[i] = vmul(vv[i], ld_keep(x + cidx[i], pl));
    unsigned fl = nv > 0 ? (bits[a >> 5] >> (a & 31)) & ((1u << nv) - 1u) : 0u;
    // a mark on the chunk's first nonzero closes the open row before it
    const bool start0 = __shfl_sync(0xffffffffu, fl & 1u, 0) != 0u;
    if (start0 && c0 > kb) {
      close_open(cval);
      crow += 1;
      c_is_first = false;
      cval = CT(0);
    }
    if (lane == 0) fl &= ~1u;
    // row of the lane's first nonzero: crow + marks in the lanes before
    const int cnt = __popc(fl);
    int pre = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int o = __shfl_up_sync(0xffffffffu, pre, d);
      if (lane >= d) pre += o;
    }
    const int total = __shfl_sync(0xffffffffu, pre, 31);
    pre -= cnt;
    // lane-sequential sums split at the marks
    Ac sum, lead;
    acc_zero(sum);
    acc_zero(lead);
    int nf = 0;
#pragma unroll
    for (int i = 0; i < kRunLane; ++i) {
      if ((fl >> i) & 1u) {
        if (nf == 0) lead = sum;
        else {
          write_row(y, yrow(crow + pre + nf), alpha, beta, (X)acc_out(sum));
          dot_add(crow + pre + nf, (CT)acc_out(sum));
        }
        ++nf;
        acc_zero(sum);
      }
      if (i < nv) acc_add(sum, p[i]);
    }
    if (nf == 0) lead = sum;
    // T = leads of this lane and the following lanes up to the first lane at
    // or after it that holds a mark (that lane's lead included)
    const unsigned marks = __ballot_sync(0xffffffffu, nf > 0);
    const unsigned ge = marks & (~0u << lane);
    const int e = ge ? __ffs(ge) - 1 : 31;
    CT T = (CT)acc_carry(lead);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const CT o = __shfl_down_sync(0xffffffffu, T, d);
      if (lane + d <= e) T += o;
    }
    CT Tn = __shfl_down_sync(0xffffffffu, T, 1);
    if (lane == 31) Tn = CT(0);
    const CT T0 = __shfl_sync(0xffffffffu, T, 0);
    if (marks == 0u) {
      cval += T0;  // the open row runs through the whole chunk
      continue;
    }
    // the open row closes at the first mark
    close_open(cval + T0);
    c_is_first = false;
    // a marked lane's tail closes at the next marked lane; the last one stays open
    const int last = 31 - __clz(marks);
    const CT tailv = (CT)acc_carry(sum) + Tn;
    if (nf > 0 && lane != last) {
      write_row(y, yrow(crow + pre + nf), alpha, beta, (X)tailv);
      dot_add(crow + pre + nf, tailv);
    }
    cval = __shfl_sync(0xffffffffu, tailv, last);
    crow += total;
  }
  // the open row: ends exactly at ke, or continues into the next warp
  const bool ends = (crow + 1 <= m) && (rst[crow + 1] == ke);
  if (lane == 0) {
    int c1 = -1;
    CT v1 = CT(0);
    dot_add(crow, cval);  // the open row's last piece, stored or carried
    if (ends && !(c_is_first && first_open)) {
      write_row(y, yrow(crow), alpha, beta, (X)cval);
    } else if (c_is_first && first_open) {
      carry0_row = crow;
      carry0 = cval;
    } else {
      c1 = crow;
      v1 = cval;
    }
    carry_row[2 * w] = carry0_row;
    carry_val[2 * w] = carry0;
    carry_row[2 * w + 1] = c1;
    carry_val[2 * w + 1] = v1;
  }
  if constexpr (DOT) {  // the warp's partial, lanes added in a fixed order
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) dotv += __shfl_xor_sync(0xffffffffu, dotv, d);
    if (lane == 0) dot_part[w] = dotv;
  }
}

}  // namespace rvvla
