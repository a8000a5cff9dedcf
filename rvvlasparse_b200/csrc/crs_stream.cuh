// crs_stream.cuh — shared-memory-free CSR SpMV for matrices without empty
// rows (every row end is a distinct position, so row heads inside a 32-wide
// chunk are one OR-reduction of the next 32 row ends).
//
// Each warp owns a contiguous range of E nonzeros (E a multiple of 32,
// balanced by construction).  Per chunk of 32 nonzeros: coalesced value and
// column loads (L2 evict-first), x gathers (L2 evict-last), heads =
// OR over lanes of (1 << (row_end - chunk_start)), an inclusive segmented
// warp scan, and one store per row that ends in the chunk.  The row open at a
// chunk end is carried in a register; rows that cross a warp boundary leave
// (row, partial) carries that a second kernel adds in warp order.  Four chunks
// are loaded before any is reduced, to keep enough bytes in flight.
#pragma once
#include "crs_merge.cuh"

namespace rvvla {

constexpr int kStreamUnroll = 4;

// Inclusive segmented warp scan of accumulators; heads start segments.
template <class Ac>
__device__ __forceinline__ Ac acc_seg_scan(Ac v, unsigned heads, unsigned lane) {
  const unsigned below = heads & ((2u << lane) - 1u);
  const int seg_start = below ? (31 - __clz(below)) : 0;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const Ac o = acc_shfl_up(v, d);
    if ((int)lane - d >= seg_start) acc_merge(v, o);
  }
  return v;
}

template <class V, class X>
__device__ __forceinline__ auto sprod(V v, X x) { return v * x; }
template <>
__device__ __forceinline__ auto sprod<__nv_bfloat16, float>(__nv_bfloat16 v, float x) { return __bfloat162float(v) * x; }

// warp w covers nonzeros [w*E, min((w+1)*E, nnz)); wrow[w] = row of its
// first nonzero.  carry_row/carry_val: 2 slots per warp (-1 = unused).
template <class V, class X, class Ac, class CT>
__global__ void __launch_bounds__(256)
crs_stream_kernel(int m, int nnz, int E, int nwarps, const int* __restrict__ Rst, const int* __restrict__ Col,
                  const V* __restrict__ Val, const X* __restrict__ x, X* __restrict__ y, X alpha, X beta,
                  const int* __restrict__ wrow, int* __restrict__ carry_row, CT* __restrict__ carry_val,
                  const int* __restrict__ row_map) {
  const int w = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const unsigned lane = threadIdx.x & 31;
  if (w >= nwarps) return;
  const int kb = w * E;
  const int ke = min(nnz, kb + E);
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  int r = wrow[w];                         // row of the current (open) segment
  const bool first_open = Rst[r] < kb;     // first row began in an earlier warp
  bool open_is_first = true;               // the open row is the warp's first row
  Ac acc;
  acc_zero(acc);
  CT cfirst = CT(0);
  int cfirst_row = -1;
  int win = (r + 1 + (int)lane <= m) ? Rst[r + 1 + lane] : INT_MAX;  // next 32 row ends
  int wbase = r;                                                     // rows win describes: wbase+1..
  for (int k0 = kb; k0 < ke; k0 += 32 * kStreamUnroll) {
    int cidx[kStreamUnroll];
    V vv[kStreamUnroll];
#pragma unroll
    for (int u = 0; u < kStreamUnroll; ++u) {
      const int k = k0 + u * 32 + (int)lane;
      if (k < ke) {
        cidx[u] = ld_stream(Col + k, pf);
        vv[u] = ld_stream(Val + k, pf);
      }
    }
    X xv[kStreamUnroll];
#pragma unroll
    for (int u = 0; u < kStreamUnroll; ++u) {
      const int k = k0 + u * 32 + (int)lane;
      if (k < ke) xv[u] = ld_keep(x + cidx[u], pl);
    }
#pragma unroll
    for (int u = 0; u < kStreamUnroll; ++u) {
      const int c0 = k0 + u * 32;
      if (c0 >= ke) break;
      const int k = c0 + (int)lane;
      const bool valid = k < ke;
      // refresh the window when its rows are used up (>= 1 row end per row)
      if (r - wbase >= 1) {
        const int shift = r - wbase;
        if (shift < 32) {
          const int nw = __shfl_down_sync(0xffffffffu, win, shift);
          const int idx = r + 1 + (int)lane;
          win = ((int)lane + shift < 32) ? nw : ((idx <= m) ? Rst[idx] : INT_MAX);
        } else {
          const int idx = r + 1 + (int)lane;
          win = (idx <= m) ? Rst[idx] : INT_MAX;
        }
        wbase = r;
      }
      // heads: element c0+i starts a new row when a row ends at c0+i.  r is
      // the row of element c0-1 (of kb for the first chunk, whose row ends
      // after kb), so a head at i = 0 means the open row ended at c0.
      const int d = win - c0;
      const unsigned bit = (d >= 0 && d < 32) ? (1u << d) : 0u;
      const unsigned heads = __reduce_or_sync(0xffffffffu, bit);
      if (heads & 1u) {  // the open row is complete before this chunk
        if (lane == 0) {
          if (open_is_first && first_open) {
            cfirst = acc_carry(acc);
            cfirst_row = r;
          } else {
            write_row(y, row_map ? row_map[r] : r, alpha, beta, (X)acc_out(acc));
          }
        }
        acc_zero(acc);
      }
      Ac p;
      acc_zero(p);
      if (valid) acc_add(p, sprod(vv[u], xv[u]));
      Ac s = acc_seg_scan(p, heads, lane);
      const unsigned upto = heads & ((2u << lane) - 1u);
      const int rel = __popc(upto);
      // the open row's earlier partial joins segment 0
      if (rel == 0) acc_merge(s, acc);
      const int last_valid = min(31, ke - 1 - c0);
      const bool next_head = ((int)lane < 31) && ((heads >> (lane + 1)) & 1u);
      const bool seg_end = valid && ((int)lane == last_valid || next_head);
      const int row = r + rel;
      // segment 0 continues the open row; when that row is the warp's first
      // row and began in an earlier warp, its piece becomes a carry (kept
      // warp-uniform: lane 0 publishes the carry slots)
      const bool first_piece_ends = !(heads & 1u) && heads != 0u && (__ffs(heads) - 1) <= last_valid &&
                                    open_is_first && first_open;
      if (first_piece_ends) {
        const CT v0 = acc_carry(acc_bcast(s, __ffs(heads) - 2));
        cfirst = v0;
        cfirst_row = r;
      }
      // a segment that ends before the chunk's last valid lane ends its row
      if (seg_end && (int)lane < last_valid && !(rel == 0 && first_piece_ends))
        write_row(y, row_map ? row_map[row] : row, alpha, beta, (X)acc_out(s));
      // the segment at the last valid lane stays open
      const Ac tailv = acc_bcast(s, last_valid);
      const unsigned nh = __popc(heads & ((2u << last_valid) - 1u));
      if (nh) open_is_first = false;
      r += nh;
      acc = tailv;
    }
  }
  // the open row: ends exactly at ke, or continues into the next warp
  const bool ends = (r + 1 <= m) && (Rst[r + 1] == ke);
  if (lane == 0) {
    int c1 = -1;
    CT v1 = CT(0);
    if (ends && !(open_is_first && first_open)) {
      write_row(y, row_map ? row_map[r] : r, alpha, beta, (X)acc_out(acc));
    } else if (open_is_first && first_open) {
      // one piece: the warp's first row is still open (or ends at ke)
      cfirst = acc_carry(acc);
      cfirst_row = r;
    } else {
      c1 = r;
      v1 = acc_carry(acc);
    }
    carry_row[2 * w] = cfirst_row;
    carry_val[2 * w] = cfirst;
    carry_row[2 * w + 1] = c1;
    carry_val[2 * w + 1] = v1;
  }
}

// Rows that cross warp boundaries: every piece is a carry (no warp wrote the
// row), so the run of equal rows is summed in warp order and written once.
template <class X, class CT>
__global__ void crs_stream_fixup_kernel(int nslots, const int* __restrict__ carry_row,
                                        const CT* __restrict__ carry_val, X* __restrict__ y, X alpha, X beta,
                                        const int* __restrict__ row_map) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nslots) return;
  const int r = carry_row[t];
  if (r < 0) return;
  int prev = t - 1;
  while (prev >= 0 && carry_row[prev] < 0) --prev;
  if (prev >= 0 && carry_row[prev] == r) return;
  CT s = carry_val[t];
  for (int u = t + 1; u < nslots; ++u) {
    const int ru = carry_row[u];
    if (ru < 0) continue;
    if (ru != r) break;
    s += carry_val[u];
  }
  const X o = alpha * (X)s;
  const int ro = row_map ? row_map[r] : r;
  y[ro] = (beta == X(0)) ? o : o + beta * y[ro];
}

__global__ void crs_stream_plan_kernel(int m, int nnz, const int* __restrict__ Rst, int E, int nwarps,
                                       int* __restrict__ wrow, int* __restrict__ any_empty);

}  // namespace rvvla
