// hcsr_spmv.cu — y = alpha*A*x + beta*y for spMtxHCSR on sm_100a.
//
// Reference: src/scalar/spmv_mtx_hcsr.cpp:22-134.  The reference walks a
// block row's blocks in block-column order and adds every block's
// contribution into y[block row]: a CSR block (kind 1) adds one row sum per
// row, a COO block (any other kind) adds one product per nonzero.  Any R and
// C are accepted (the only limits are the format's: uint16 local columns,
// 30-bit row_ptr offsets).
//
// GPU mapping.  One CTA of 16 warps per block row; the block row's R partial
// sums live in shared memory (or, for block rows too tall for shared memory,
// in a global scratch slice the CTA owns).  Every row belongs to one warp:
// warp w owns rows [ceil(w*rows/16), ceil((w+1)*rows/16)), so no two warps
// ever add into the same row and the summation order of every row is fixed —
// the result is bitwise reproducible run to run (no float atomics).
//
// The block columns are taken in windows of kHWin blocks: the window's
// non-empty blocks are compacted into a row-range list and a COO list in
// shared memory (so the metadata staged never depends on b_n), then
//   * row-range phase: each warp walks, in block order, every CSR block and
//     every COO block of at least kHBig nonzeros for its own rows.  A CSR
//     block's nonzeros of those rows are one contiguous range, streamed in
//     chunks of 256 (8 consecutive nonzeros per lane, 16-byte loads of values
//     and uint16 columns); the rows starting inside a chunk are marked from
//     the block's row_ptr (a window of 32 row starts per lane set, loaded one
//     window ahead), each lane sums its 8 products split at the marks, and a
//     reverse segmented warp scan closes the rows that cross lanes, so each
//     row piece of a chunk is added to the accumulator exactly once.  A large
//     COO block keeps its nonzeros in row order (the builder writes them so):
//     the warp finds its range by a 32-ary search on the rows and streams it
//     the same way, a row starting wherever the row changes; a CTA that finds
//     rows out of order there starts its block row over with every COO block
//     in the COO phase;
//   * COO phase: the window's other COO nonzeros (in block order) are cut
//     into rounds of 1024; every warp computes 64 products in stream order
//     (the block of each nonzero from the compacted list: a warp-wide OR of
//     the next block starts and a popcount), writes (row, product, owner) to
//     shared memory — a run of one row inside one block summed first, by a
//     segmented warp scan — and after a barrier each owner warp picks its own
//     run sums in stream order and adds them 32 at a time (COO rows belong to
//     warps in interleaved chunks of 16 rows, so that the few hundred
//     consecutive rows of a block spread over the warps; the row-range
//     phase's ranges are not needed here, since barriers separate the
//     phases); lanes holding the same row add one after another in lane
//     order (an integer atomicMin over a per-warp slot table elects the
//     lowest pending lane of each row per round).
// The next round's loads are issued before the current round is applied.
// A COO row index at or beyond the block row's rows (malformed input; the
// builder never writes one) is skipped rather than written out of range.
// Per row, the sum is: row-range pieces of window 0 in block order, COO
// products of window 0 in stream order, then window 1, ...; y = alpha*acc +
// beta*y at the end (y is not read when beta == 0).  Shared memory is sized
// for two CTAs per SM and the carveout asks for no more, so that the rest of
// the SM's 256 KB serves as L1 for the gathers of x.
//
// Mixed forms: lane sums of the CSR phase in compensated fp32 (two-sum), COO
// products in fp32; the block-row accumulator, where pieces of different
// blocks meet, is fp64.
#include <algorithm>
#include <cstring>
#include <string>
#include <type_traits>

#include "crs_merge.cuh"
#include "crs_run.cuh"
#include "rvvla_internal.cuh"

namespace rvvla {
namespace {

constexpr uint32_t kHKindMask = 0x3FFFFFFFu;
constexpr int kHW = 16;                    // warps per CTA = row owners
constexpr int kHT = 32 * kHW;              // threads per CTA
constexpr int kHMinBlocks = 2;             // resident CTAs per SM the registers are sized for
constexpr int kHWLog = kHW == 8 ? 3 : 4;
static_assert(kHW == 8 || kHW == 16, "8 or 16 row owners");
constexpr int kHPer = 1;                   // block columns per thread in a window
constexpr int kHWin = kHPer * kHT;         // block columns per window
constexpr int kHRound = 1024;              // COO nonzeros per round
constexpr int kHU = kHRound / (kHW * 32);  // sub-steps of 32 per warp and round
constexpr int kHStages = 2;                // COO stage buffers (round t fills t % kHStages)
constexpr int kHSlots = 2048 / kHW;        // per-warp row slots of the COO apply (power of two)
constexpr int kHBig = 1024;                // COO blocks of at least this many nonzeros take the row-range path
constexpr int kHLane = 8;                  // CSR nonzeros per lane and chunk
constexpr int kHChunk = 32 * kHLane;
constexpr int kHWscr = kHChunk * 4 > 1024 ? kHChunk * 4 : 1024;  // per-warp scratch bytes

// a non-empty block of the window: COO stream start (COO list only), nonzero
// offset, row_ptr offset, block column
struct HBlk {
  int cs;
  int bp;
  uint32_t off;
  int j;
};
static_assert(sizeof(HBlk) == 16, "HBlk is one 16-byte shared-memory load");

__host__ __device__ constexpr size_t hal16(size_t b) { return (b + 15) / 16 * 16; }

// Dynamic shared memory: [acc] list | prod | row | own | per-warp scratch |
// per-warp mark groups.
template <class SA, class P>
struct HLayout {
  size_t acc, list, prod, row, own, wscr, mgrp, slot, total;
  __host__ __device__ explicit HLayout(int64_t racc) {
    acc = 0;
    list = hal16((size_t)racc * sizeof(SA));
    prod = list + hal16((size_t)(kHWin + 1) * sizeof(HBlk));
    row = prod + hal16((size_t)kHStages * kHRound * sizeof(P));
    own = row + (size_t)kHStages * kHRound * 4;
    wscr = own + hal16((size_t)kHStages * kHRound);
    mgrp = wscr + (size_t)kHW * kHWscr;
    slot = mgrp + (size_t)kHW * 32 * 4;
    total = slot + (size_t)kHW * kHSlots * 4;
  }
};

template <class V, class X, class SA, bool MIX>
struct HTypes {
  using Ac = std::conditional_t<MIX, CompF32, SA>;  // CSR lane sums
  using P = SA;                                     // a COO run sum (fp64 in the mixed forms)
  using PT = decltype(vmul(V(), X()));              // a product
};

// COO rows belong to warps in chunks of 16 consecutive rows, interleaved
// (a block of a few hundred consecutive rows spreads over the warps)
__device__ __forceinline__ uint32_t hcsr_coo_owner(uint32_t r) { return (r >> 4) & (kHW - 1); }
// the slot of an owned row in its warp's table: distinct for 16 * kHSlots
// consecutive rows
__device__ __forceinline__ uint32_t hcsr_coo_slot(uint32_t r) {
  return (((r >> (4 + kHWLog)) << 4) | (r & 15)) & (kHSlots - 1);
}

// Exclusive CTA-wide scan of three counters; t* are the CTA totals.
__device__ __forceinline__ void hcsr_scan3(int a, int b, int c, int& pa, int& pb, int& pc, int& ta, int& tb,
                                           int& tc, int* s_w) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int ia = a, ib = b, ic = c;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int oa = __shfl_up_sync(0xffffffffu, ia, d);
    const int ob = __shfl_up_sync(0xffffffffu, ib, d);
    const int oc = __shfl_up_sync(0xffffffffu, ic, d);
    if (lane >= d) {
      ia += oa;
      ib += ob;
      ic += oc;
    }
  }
  if (lane == 31) {
    s_w[warp] = ia;
    s_w[kHW + warp] = ib;
    s_w[2 * kHW + warp] = ic;
  }
  __syncthreads();
  int wa = 0, wb = 0, wc = 0;
  ta = tb = tc = 0;
#pragma unroll
  for (int w = 0; w < kHW; ++w) {
    const int va = s_w[w], vb = s_w[kHW + w], vc = s_w[2 * kHW + w];
    if (w < warp) {
      wa += va;
      wb += vb;
      wc += vc;
    }
    ta += va;
    tb += vb;
    tc += vc;
  }
  pa = wa + ia - a;
  pb = wb + ib - b;
  pc = wc + ic - c;
  __syncthreads();
}

// eight uint16 columns with one 16-byte load
// kHLane uint16 columns with 16-byte loads
__device__ __forceinline__ void hcsr_cols(const uint16_t* p, uint32_t (&c)[kHLane], uint64_t pol) {
#pragma unroll
  for (int h = 0; h < kHLane / 8; ++h) {
    const int4 t = ld_v4_l1(p + 8 * h, pol);
    const uint32_t w[4] = {(uint32_t)t.x, (uint32_t)t.y, (uint32_t)t.z, (uint32_t)t.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      c[8 * h + 2 * q] = w[q] & 0xFFFFu;
      c[8 * h + 2 * q + 1] = w[q] >> 16;
    }
  }
}

// kHLane values with 16-byte loads
template <class V>
__device__ __forceinline__ void hcsr_vals(const V* p, V (&v)[kHLane], uint64_t pol) {
  constexpr int E = 16 / (int)sizeof(V);  // values per load
#pragma unroll
  for (int q = 0; q < kHLane / E; ++q) {
    const int4 t = ld_v4_l1(p + E * q, pol);
    V tmp[E];
    static_assert(sizeof(tmp) == sizeof(int4), "one 16-byte load");
    memcpy(tmp, &t, sizeof(int4));
#pragma unroll
    for (int e = 0; e < E; ++e) v[E * q + e] = tmp[e];
  }
}

template <class V>
__device__ __forceinline__ V hcsr_ld1(const V* p) {
  if constexpr (std::is_same_v<V, __nv_bfloat16>) return __ushort_as_bfloat16(__ldg((const unsigned short*)p));
  else return __ldg(p);
}

template <class SA, class T>
__device__ __forceinline__ void hcsr_add(SA* acc, int r, T v) {
  acc[r] += (SA)v;
}

// Row-range phase of one warp for one CSR block: the nonzeros of the warp's
// rows [ra, rb).  Chunks of kHChunk nonzeros, kHLane consecutive ones per
// lane (16-byte loads): positions count from the block's first nonzero
// rounded down to a multiple of 8, so a chunk start is 16-byte aligned
// whenever the arrays are (VEC).  Row starts come from the block's row_ptr
// in windows of 32 rows (the next window loaded one window ahead) and mark
// the lanes' slots through a per-warp table; each lane sums its products
// split at the marks, and a reverse segmented scan adds the parts of rows
// crossing lanes.  When no lane holds two row starts (rows of 8 or more
// nonzeros), a lane's sums take the short split at its one mark.  The
// columns of a chunk are loaded one chunk ahead, so that its x gathers leave
// together with its value loads.
template <class V, class X, class SA, bool MIX, bool VEC>
__device__ __forceinline__ void hcsr_csr_rows(const uint32_t* __restrict__ rp, int64_t bp, int ra, int rb, int64_t nz,
                                              const uint16_t* __restrict__ col_idx, const V* __restrict__ values,
                                              const X* __restrict__ xb, SA* acc, int* table, uint32_t* mgrp, int lane,
                                              uint64_t pf, uint64_t pl) {
  using Ty = HTypes<V, X, SA, MIX>;
  using Ac = typename Ty::Ac;
  using PT = typename Ty::PT;
  using CT = SA;
  const int64_t base = bp & ~(int64_t)7;
  const uint32_t off = (uint32_t)(bp - base);
  const uint32_t lo = off + __ldg(rp + ra), hi = off + __ldg(rp + rb);
  if (lo >= hi) return;
  const uint32_t lim = (uint32_t)(nz - base);  // positions below lim lie inside the arrays
  const V* __restrict__ vb = values + base;
  const uint16_t* __restrict__ cb = col_idx + base;
  int wb = ra;
  auto ldwin = [&](int b0, uint32_t& s, uint32_t& e) {
    const int r = b0 + lane;
    s = r < rb ? off + __ldg(rp + r) : 0xFFFFFFFFu;
    e = r < rb ? off + __ldg(rp + r + 1) : 0xFFFFFFFFu;
  };
  uint32_t s_c, e_c, s_n, e_n;
  ldwin(wb, s_c, e_c);
  ldwin(wb + 32, s_n, e_n);
  int open_row = -1;
  // the lane's 8 columns of the next chunk, loaded one chunk ahead, so that
  // a chunk's x gathers leave together with its value loads
  const uint32_t c0 = lo & ~7u;
  int4 cn = make_int4(0, 0, 0, 0);
  if (VEC && c0 + kHLane * lane + kHLane <= lim) cn = ld_v4_l1(cb + c0 + kHLane * lane, pf);
  for (uint32_t c = c0; c < hi; c += kHChunk) {
    const uint32_t a = c + kHLane * lane;
    const uint32_t fv = lo > a ? lo - a : 0u;  // the lane's slots in [fv, lv) lie in [lo, hi)
    const uint32_t lv = hi > a ? hi - a : 0u;
    const int4 cw = cn;
    if (VEC) {
      const uint32_t an = a + kHChunk;
      cn = c + kHChunk < hi && an + kHLane <= lim ? ld_v4_l1(cb + an, pf) : make_int4(0, 0, 0, 0);
    }
    // ---- loads and products
    PT p[kHLane];
    {
      V vv[kHLane];
      uint32_t cc[kHLane];
      if (VEC && a + kHLane <= lim) {
        hcsr_vals(vb + a, vv, pf);
        const uint32_t w[4] = {(uint32_t)cw.x, (uint32_t)cw.y, (uint32_t)cw.z, (uint32_t)cw.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          cc[2 * q] = w[q] & 0xFFFFu;
          cc[2 * q + 1] = w[q] >> 16;
        }
      } else {
#pragma unroll
        for (int i = 0; i < kHLane; ++i) {
          const bool in = a + i < lim;
          vv[i] = in ? hcsr_ld1(vb + a + i) : V(0);
          cc[i] = in ? (uint32_t)__ldg(cb + a + i) : 0u;
        }
      }
#pragma unroll
      for (int i = 0; i < kHLane; ++i) {
        const bool ok = (uint32_t)i >= fv && (uint32_t)i < lv;
        if constexpr (MIX) p[i] = ok ? to_f32(vv[i]) * (float)ld_keep(xb + cc[i], pl) : 0.f;
        else p[i] = ok ? vv[i] * ld_keep(xb + cc[i], pl) : PT(0);
      }
    }
    // ---- marks of the rows that start inside the chunk
    mgrp[lane] = 0u;
    __syncwarp();
    for (;;) {
      const uint32_t pos = s_c - c;  // wraps for rows that started before the chunk
      if (pos < (uint32_t)kHChunk && s_c < e_c) {
        table[pos] = wb + lane;
        atomicOr(mgrp + pos / kHLane, 1u << (pos % kHLane));
      }
      const uint32_t s31 = __shfl_sync(0xffffffffu, s_c, 31);
      if (!(wb + 32 < rb && s31 < c + kHChunk)) break;
      wb += 32;
      s_c = s_n;
      e_c = e_n;
      ldwin(wb + 32, s_n, e_n);
    }
    __syncwarp();
    const uint32_t mb = mgrp[lane];
    // ---- lane sums: lead = before the lane's first mark, sum = from its last
    // mark; rows that start and end inside the lane are added now
    Ac sum, lead;
    acc_zero(sum);
    acc_zero(lead);
    int nf = 0, rcur = -1;
    if (!__any_sync(0xffffffffu, (mb & (mb - 1u)) != 0u)) {
      const int m = mb ? __ffs(mb) - 1 : kHLane;
#pragma unroll
      for (int i = 0; i < kHLane; ++i) {
        if (i == m) {
          lead = sum;
          acc_zero(sum);
        }
        acc_add(sum, p[i]);
      }
      if (mb) {
        nf = 1;
        rcur = table[kHLane * lane + m];
      } else {
        lead = sum;
      }
    } else {
#pragma unroll
      for (int i = 0; i < kHLane; ++i) {
        if ((mb >> i) & 1u) {
          if (nf == 0) lead = sum;
          else hcsr_add(acc, rcur, acc_carry(sum));
          rcur = table[kHLane * lane + i];
          ++nf;
          acc_zero(sum);
        }
        acc_add(sum, p[i]);
      }
      if (nf == 0) lead = sum;
    }
    // ---- rows crossing lanes: reverse segmented scan of the leads
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
    if (lane == 0 && open_row >= 0) hcsr_add(acc, open_row, T0);
    if (nf > 0) hcsr_add(acc, rcur, (CT)acc_carry(sum) + Tn);
    if (marks) open_row = __shfl_sync(0xffffffffu, rcur, 31 - __clz(marks));
    __syncwarp();
  }
}

// First k in [0, cnt) with rows[k] >= t (cnt when none), for ascending rows;
// a 32-ary search of the warp (each step probes 32 positions).  On rows that
// do not ascend the result is some k in [0, cnt].
__device__ __forceinline__ int hcsr_lower_bound(const uint32_t* __restrict__ rows, int cnt, uint32_t t, int lane) {
  int lo = 0, hi = cnt;  // the answer lies in [lo, hi]
  while (hi - lo > 32) {
    const int k = lo + (int)(((int64_t)(hi - lo) * lane) >> 5);
    const int c = __popc(__ballot_sync(0xffffffffu, __ldg(rows + k) < t));
    const int nlo = c > 0 ? __shfl_sync(0xffffffffu, k, (c - 1) & 31) + 1 : lo;
    const int nhi = c < 32 ? __shfl_sync(0xffffffffu, k, c & 31) : hi;
    lo = nlo;
    hi = max(nhi, nlo);
  }
  const bool less = lo + lane < hi && __ldg(rows + lo + lane) < t;
  return lo + __popc(__ballot_sync(0xffffffffu, less));
}

// Row-range phase of one warp for one large COO block: the nonzeros
// [lo, hi) (absolute) that hold the warp's rows [ra, rb), in chunks of 256 as
// in hcsr_csr_rows.  rp holds each nonzero's row (rp[k - bp]); a row starts
// where the row differs from the previous kept nonzero's.  Returns true when
// a row descends or lies outside [ra, rb); such nonzeros are left out.
template <class V, class X, class SA, bool MIX, bool VEC>
__device__ __forceinline__ bool hcsr_coo_rows(const uint32_t* __restrict__ rp, int64_t bp, int ra, int rb, int64_t lo,
                                              int64_t hi, int64_t nz, const uint16_t* __restrict__ col_idx,
                                              const V* __restrict__ values, const X* __restrict__ xb, SA* acc,
                                              int lane, uint64_t pf, uint64_t pl) {
  using Ty = HTypes<V, X, SA, MIX>;
  using Ac = typename Ty::Ac;
  using PT = typename Ty::PT;
  using CT = SA;
  uint32_t last_row = 0xFFFFFFFFu;   // row of the last nonzero before the chunk
  uint32_t last_kept = 0xFFFFFFFFu;  // the same, of the kept nonzeros
  bool bad = false;
  int open_row = -1;
  for (int64_t c = lo & ~(int64_t)7; c < hi; c += kHChunk) {
    const int64_t a = c + kHLane * lane;
    // ---- rows (0xFFFFFFFF outside [lo, hi) and outside [ra, rb))
    uint32_t rw[kHLane];
    {
#pragma unroll
      for (int i = 0; i < kHLane; ++i) rw[i] = a + i >= lo && a + i < hi ? __ldg(rp + (a + i - bp)) : 0xFFFFFFFFu;
      uint32_t before = __shfl_up_sync(0xffffffffu, rw[kHLane - 1], 1);
      if (lane == 0) before = last_row;
      const uint32_t l31 = __shfl_sync(0xffffffffu, rw[kHLane - 1], 31);
      last_row = l31 != 0xFFFFFFFFu ? l31 : last_row;
#pragma unroll
      for (int i = 0; i < kHLane; ++i) {
        if (rw[i] != 0xFFFFFFFFu) {
          if ((before != 0xFFFFFFFFu && rw[i] < before) || rw[i] < (uint32_t)ra || rw[i] >= (uint32_t)rb) bad = true;
          before = rw[i];
          if (rw[i] < (uint32_t)ra || rw[i] >= (uint32_t)rb) rw[i] = 0xFFFFFFFFu;
        }
      }
    }
    // ---- loads and products
    PT p[kHLane];
    {
      V vv[kHLane];
      uint32_t cc[kHLane];
      const bool any = a < hi && a + kHLane > lo;
      if (VEC && any && a + kHLane <= nz) {
        hcsr_vals(values + a, vv, pf);
        hcsr_cols(col_idx + a, cc, pf);
      } else {
#pragma unroll
        for (int i = 0; i < kHLane; ++i) {
          const bool ok = a + i >= lo && a + i < hi;
          vv[i] = ok ? hcsr_ld1(values + a + i) : V(0);
          cc[i] = ok ? (uint32_t)__ldg(col_idx + a + i) : 0u;
        }
      }
#pragma unroll
      for (int i = 0; i < kHLane; ++i) {
        const bool ok = rw[i] != 0xFFFFFFFFu;
        if constexpr (MIX) p[i] = ok ? to_f32(vv[i]) * (float)ld_keep(xb + cc[i], pl) : 0.f;
        else p[i] = ok ? vv[i] * ld_keep(xb + cc[i], pl) : PT(0);
      }
    }
    // ---- marks of the rows that start inside the chunk
    uint32_t mb = 0;
    {
      // a row starts where it differs from the previous kept nonzero's
      uint32_t prev = __shfl_up_sync(0xffffffffu, rw[kHLane - 1], 1);
      if (lane == 0) prev = last_kept;
#pragma unroll
      for (int i = 0; i < kHLane; ++i) {
        const uint32_t before = i == 0 ? prev : rw[i - 1];
        if (rw[i] != 0xFFFFFFFFu && rw[i] != before) mb |= 1u << i;
      }
      const uint32_t k31 = __shfl_sync(0xffffffffu, rw[kHLane - 1], 31);
      last_kept = k31 != 0xFFFFFFFFu ? k31 : last_kept;
    }
    // ---- lane sums split at the marks; rows closed inside the lane are added now
    Ac sum, lead;
    acc_zero(sum);
    acc_zero(lead);
    int nf = 0, rcur = -1;
#pragma unroll
    for (int i = 0; i < kHLane; ++i) {
      if ((mb >> i) & 1u) {
        if (nf == 0) lead = sum;
        else hcsr_add(acc, rcur, acc_carry(sum));
        rcur = (int)rw[i];
        ++nf;
        acc_zero(sum);
      }
      acc_add(sum, p[i]);
    }
    if (nf == 0) lead = sum;
    // ---- rows crossing lanes: reverse segmented scan of the leads
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
    if (lane == 0 && open_row >= 0) hcsr_add(acc, open_row, T0);
    if (nf > 0) hcsr_add(acc, rcur, (CT)acc_carry(sum) + Tn);
    if (marks) open_row = __shfl_sync(0xffffffffu, rcur, 31 - __clz(marks));
    __syncwarp();
  }
  return bad;
}

// Raw loads of one COO sub-step (32 consecutive COO nonzeros of the window).
template <class V>
struct HCooRaw {
  uint32_t row;
  uint32_t col;
  V v;
  int64_t xoff;
  bool ok;
};

template <class V, class X, class SA, bool MIX, bool VEC, bool GACC>
__global__ void __launch_bounds__(kHT, kHMinBlocks)
hcsr_spmv_kernel(int64_t R, int64_t C, int64_t m, int64_t nz, int64_t b_n, const int* __restrict__ block_ptr,
                 const uint32_t* __restrict__ row_offset, const uint32_t* __restrict__ row_ptr,
                 const uint16_t* __restrict__ col_idx, const V* __restrict__ values, const X* __restrict__ x,
                 X* __restrict__ y, X alpha, X beta, SA* __restrict__ gacc) {
  using Ty = HTypes<V, X, SA, MIX>;
  using P = typename Ty::P;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_w[3 * kHW];
  const HLayout<SA, P> L(GACC ? 0 : R);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t br = blockIdx.x;
  const int64_t r0 = br * R;
  const int rows = (int)min(R, m - r0);
  SA* acc = GACC ? gacc + r0 : reinterpret_cast<SA*>(smem + L.acc);
  HBlk* list = reinterpret_cast<HBlk*>(smem + L.list);
  P* s_prod0 = reinterpret_cast<P*>(smem + L.prod);
  uint32_t* s_row0 = reinterpret_cast<uint32_t*>(smem + L.row);
  uint8_t* s_own0 = smem + L.own;
  int* table = reinterpret_cast<int*>(smem + L.wscr + (size_t)warp * kHWscr);          // CSR phase
  uint16_t* olist = reinterpret_cast<uint16_t*>(smem + L.wscr + (size_t)warp * kHWscr);  // COO phase
  uint32_t* mgrp = reinterpret_cast<uint32_t*>(smem + L.mgrp) + warp * 32;
  __shared__ int s_bad;  // a large COO block whose rows do not ascend was met
  bool big_ok = true;
  int* slot = reinterpret_cast<int*>(smem + L.slot) + warp * kHSlots;
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();

  for (int li = tid; li < rows; li += kHT) acc[li] = SA(0);
  for (int q = lane; q < kHSlots; q += 32) slot[q] = INT_MAX;
  if (tid == 0) s_bad = 0;
  // this warp's rows
  const int ra = (int)(((int64_t)warp * rows + kHW - 1) / kHW);
  const int rb = (int)(((int64_t)(warp + 1) * rows + kHW - 1) / kHW);
  const int64_t blk0 = br * b_n;
  __syncthreads();

  for (;;) {
  for (int64_t jw = 0; jw < b_n; jw += kHWin) {
    const int nb = (int)(b_n - jw < kHWin ? b_n - jw : kHWin);
    // ---- compact the window's non-empty blocks (kHPer consecutive per thread):
    // CSR blocks and COO blocks of >= kHBig nonzeros form the row-range list
    // (block order, from the back of `list`), the smaller COO blocks the COO
    // stream (from the front, with a sentinel)
    int bpq[kHPer], cntq[kHPer];
    uint32_t roq[kHPer];
    int kindq[kHPer];  // 0 none, 1 CSR, 2 large COO, 3 small COO
#pragma unroll
    for (int q = 0; q < kHPer; ++q) {
      const int jj = kHPer * tid + q;
      bpq[q] = 0;
      cntq[q] = 0;
      roq[q] = 0u;
      kindq[q] = 0;
      if (jj < nb) {
        const int64_t b = blk0 + jw + jj;
        bpq[q] = block_ptr[b];
        cntq[q] = block_ptr[b + 1] - bpq[q];
        roq[q] = row_offset[b];
        if (cntq[q] > 0) kindq[q] = (roq[q] >> 30) == 1u ? 1 : (cntq[q] >= kHBig && big_ok ? 2 : 3);
      }
    }
    int n_seg = 0, n_coo = 0, n_ent = 0;
#pragma unroll
    for (int q = 0; q < kHPer; ++q) {
      if (kindq[q] == 1 || kindq[q] == 2) ++n_seg;
      if (kindq[q] == 3) {
        ++n_coo;
        n_ent += cntq[q];
      }
    }
    int p_seg, p_coo, p_ent, t_seg, t_coo, t_ent;
    hcsr_scan3(n_seg, n_coo, n_ent, p_seg, p_coo, p_ent, t_seg, t_coo, t_ent, s_w);
#pragma unroll
    for (int q = 0; q < kHPer; ++q) {
      if (kindq[q] == 0) continue;
      HBlk h;
      h.bp = bpq[q];
      h.off = roq[q] & kHKindMask;
      h.j = (int)(jw + kHPer * tid + q);
      if (kindq[q] == 1 || kindq[q] == 2) {
        h.cs = kindq[q] == 1 ? -1 : cntq[q];  // a large COO block keeps its nonzero count
        list[kHWin + 1 - t_seg + p_seg++] = h;
      } else {
        h.cs = p_ent;
        p_ent += cntq[q];
        list[p_coo++] = h;
      }
    }
    if (tid == 0) list[t_coo].cs = t_ent;  // sentinel: end of the COO stream
    __syncthreads();

    // ---- row-range phase: this warp's rows of every CSR block and large
    // COO block of the window, in block order.  A large COO block's rows
    // ascend (the builder writes them so): the warp finds its nonzeros
    // [first row >= ra, first row >= rb) by search and checks, on the way,
    // that they ascend and lie in [ra, rb); a CTA whose warps met anything
    // else redoes its block row with every COO block in the COO stream.
    for (int i = 0; i < t_seg; ++i) {
      const HBlk h = list[kHWin + 1 - t_seg + i];
      const uint32_t* rp = row_ptr + h.off;
      if (h.cs < 0) {
        if (ra >= rb) continue;
        hcsr_csr_rows<V, X, SA, MIX, VEC>(rp, h.bp, ra, rb, nz, col_idx, values, x + (int64_t)h.j * C, acc, table,
                                          mgrp, lane, pf, pl);
      } else {
        const int cnt = h.cs;
        const int klo = warp == 0 ? 0 : hcsr_lower_bound(rp, cnt, (uint32_t)ra, lane);
        const int khi = warp == kHW - 1 ? cnt : hcsr_lower_bound(rp, cnt, (uint32_t)rb, lane);
        if (klo > khi) {
          if (lane == 0) s_bad = 1;
          continue;
        }
        if (klo == khi) continue;
        if (hcsr_coo_rows<V, X, SA, MIX, VEC>(rp, h.bp, ra, rb, (int64_t)h.bp + klo, (int64_t)h.bp + khi, nz, col_idx,
                                              values, x + (int64_t)h.j * C, acc, lane, pf, pl))
          s_bad = 1;
      }
    }

    // ---- COO phase: rounds of kHRound nonzeros of the window's COO stream
    if (t_ent > 0) {
      const int ncoo = t_coo, ntot = t_ent;
      const int nrounds = (ntot + kHRound - 1) / kHRound;
      HCooRaw<V> raw[kHU];
      auto coo_load = [&](int t) {
        const int q00 = t * kHRound + warp * (kHU * 32);
        int ia = 0;
        if (lane == 0) {
          const int qs = min(q00, ntot - 1);
          int lo = 0, hi = ncoo;
          while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (list[mid].cs <= qs) lo = mid;
            else hi = mid;
          }
          ia = lo;
        }
        ia = __shfl_sync(0xffffffffu, ia, 0);
#pragma unroll
        for (int u = 0; u < kHU; ++u) {
          const int q0 = q00 + 32 * u;
          const int nxt = ia + 1 + lane;
          const int d = nxt <= ncoo ? list[nxt].cs - q0 : 32;
          const unsigned mask = __reduce_or_sync(0xffffffffu, (d >= 0 && d < 32) ? 1u << d : 0u);
          int blk = ia + __popc(mask & ((2u << lane) - 1u));
          blk = min(blk, ncoo - 1);
          const int q = q0 + lane;
          HCooRaw<V>& r = raw[u];
          r.ok = q < ntot;
          r.row = 0u;
          r.xoff = -1;
          if (r.ok) {
            const HBlk h = list[blk];
            const int e = q - h.cs;
            const int64_t k = (int64_t)h.bp + e;
            r.row = ld_stream(row_ptr + h.off + e, pf);
            r.col = (uint32_t)ld_stream(col_idx + k, pf);
            r.v = ld_stream(values + k, pf);
            r.xoff = (int64_t)h.j * C;
            r.ok = r.row < (uint32_t)rows;  // a row beyond the block row (malformed input) is skipped
          }
          ia = __shfl_sync(0xffffffffu, blk, 31);
        }
      };
      coo_load(0);
      for (int t = 0; t < nrounds; ++t) {
        // this round's stage buffer: with two, round t + 1 is produced while
        // slower warps still apply round t, and one barrier per round does
        P* const s_prod = s_prod0 + (t % kHStages) * kHRound;
        uint32_t* const s_row = s_row0 + (t % kHStages) * kHRound;
        uint8_t* const s_own = s_own0 + (t % kHStages) * kHRound;
        // products of this round into shared memory, in stream order
        X xv[kHU];
#pragma unroll
        for (int u = 0; u < kHU; ++u) xv[u] = raw[u].ok ? ld_keep(x + raw[u].xoff + raw[u].col, pl) : X(0);
#pragma unroll
        for (int u = 0; u < kHU; ++u) {
          const int i = warp * (kHU * 32) + 32 * u + lane;
          const HCooRaw<V>& r = raw[u];
          P pv = P(0);
          if (r.ok) {
            if constexpr (MIX) pv = (P)(to_f32(r.v) * (float)xv[u]);
            else pv = (P)(r.v * xv[u]);
          }
          // runs of one row inside one block (consecutive lanes) are summed
          // here; only the run's last lane is handed on
          // (cont: this lane continues the previous lane's run; most
          // sub-steps have none, and skip the scan)
          const uint32_t prow = __shfl_up_sync(0xffffffffu, r.row, 1);
          const int64_t pxo = __shfl_up_sync(0xffffffffu, r.xoff, 1);
          const bool cont = lane > 0 && r.ok && prow == r.row && pxo == r.xoff;
          P run = pv;
          bool tail = r.ok;
          if (__any_sync(0xffffffffu, cont)) {
            run = warp_seg_scan(pv, !cont, lane);
            const bool ncont = __shfl_down_sync(0xffffffffu, cont, 1);
            tail = r.ok && (lane == 31 || !ncont);
          }
          s_prod[i] = run;
          s_row[i] = r.row;
          s_own[i] = (uint8_t)(tail ? hcsr_coo_owner(r.row) : 0xFFu);
        }
        __syncthreads();
        if (t + 1 < nrounds) coo_load(t + 1);
        // this warp's nonzeros of the round, in stream order
        const uint32_t me = (uint32_t)warp * 0x01010101u;
#pragma unroll 1
        for (int it = 0; it < kHRound / 512; ++it) {
          const uint4 w4 = reinterpret_cast<const uint4*>(s_own)[it * 32 + lane];
          const uint32_t ws[4] = {w4.x, w4.y, w4.z, w4.w};
          uint32_t m16 = 0;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const uint32_t eq = __vcmpeq4(ws[q], me);
            m16 |= (((eq >> 7) & 1u) | ((eq >> 14) & 2u) | ((eq >> 21) & 4u) | ((eq >> 28) & 8u)) << (4 * q);
          }
          const int cnt = __popc(m16);
          int inc = cnt;
#pragma unroll
          for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc += o;
          }
          const int total = __shfl_sync(0xffffffffu, inc, 31);
          int pos = inc - cnt;
          while (m16) {
            const int b = __ffs(m16) - 1;
            olist[pos++] = (uint16_t)(it * 512 + 16 * lane + b);
            m16 &= m16 - 1u;
          }
          __syncwarp();
          // groups of 32 of this warp's nonzeros; inside a group, rounds in
          // which the lowest pending lane of every row slot adds its value
          // (an integer atomicMin elects it), so each row receives its
          // values in lane order = stream order, whatever the scheduling
          for (int g = 0; g < total; g += 32) {
            const int tt = g + lane;
            bool pend = tt < total;
            uint32_t r = 0;
            SA pv = SA(0);
            if (pend) {
              const int i = olist[tt];
              r = s_row[i];
              pv = (SA)s_prod[i];
            }
            int* sl = slot + hcsr_coo_slot(r);
            while (__ballot_sync(0xffffffffu, pend)) {
              if (pend) atomicMin(sl, lane);
              __syncwarp();
              const bool win = pend && *sl == lane;
              __syncwarp();
              if (win) {
                acc[r] += pv;
                *sl = INT_MAX;
                pend = false;
              }
              __syncwarp();
            }
          }
        }
        if (kHStages == 1) __syncthreads();
      }
    }
    __syncthreads();
  }
  if (!big_ok || !s_bad) break;
  // rows of a large COO block out of order: start over, all COO blocks
  // through the COO stream
  big_ok = false;
  __syncthreads();
  for (int li = tid; li < rows; li += kHT) acc[li] = SA(0);
  __syncthreads();
  }
  for (int li = tid; li < rows; li += kHT) {
    const X o = (X)acc[li];
    X* yp = y + r0 + li;
    *yp = (beta == X(0)) ? alpha * o : alpha * o + beta * *yp;
  }
}

int hcsr_validate(const rvvla_hcsr* A, const void* x, const void* y) {
  if (!A) return fail(RVVLA_ERR_INVALID_ARG, "hcsr: null descriptor");
  if (A->R <= 0 || A->C <= 0 || A->m < 0 || A->n < 0 || A->nz < 0)
    return fail(RVVLA_ERR_INVALID_ARG, "hcsr: bad sizes");
  if (A->b_m != (A->m + A->R - 1) / A->R || A->b_n != (A->n + A->C - 1) / A->C)
    return fail(RVVLA_ERR_FORMAT, "hcsr: b_m/b_n inconsistent with m, n, R, C");
  if (A->m > 0 && (!A->block_ptr || !A->row_offset || !y)) return fail(RVVLA_ERR_INVALID_ARG, "hcsr: null array");
  if (A->nz > 0 && (!A->col_idx || !A->values || !A->row_ptr || !x))
    return fail(RVVLA_ERR_INVALID_ARG, "hcsr: null array");
  if (A->C > 65536) return fail(RVVLA_ERR_TOO_LARGE, "hcsr: C > 65536 does not fit the uint16 col_idx");
  if (A->m > INT32_MAX || A->nz > INT32_MAX) return fail(RVVLA_ERR_TOO_LARGE, "hcsr: m or nz beyond 2^31 - 1");
  return RVVLA_OK;
}

// Largest dynamic shared memory one CTA may take (227 KB on sm_100a).
constexpr size_t kHSmemMax = 227 * 1024;

template <class V, class X, class SA, bool MIX, bool VEC, bool GACC>
int hcsr_launch(const rvvla_hcsr* A, X alpha, const X* x, X beta, X* y, SA* gacc, size_t smem, cudaStream_t st) {
  auto kern = hcsr_spmv_kernel<V, X, SA, MIX, VEC, GACC>;
  RVVLA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // shared memory for kHMinBlocks CTAs, the rest of the SM's 256 KB as L1
  // (the gathers of x hit there)
  const int carve = (int)std::min<size_t>(100, (kHMinBlocks * (smem + 1024) * 100 + kHSmemMax - 1) / kHSmemMax);
  RVVLA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
  kern<<<(unsigned)A->b_m, kHT, smem, st>>>(A->R, A->C, A->m, A->nz, A->b_n, A->block_ptr, A->row_offset,
                                            A->row_ptr, A->col_idx, (const V*)A->values, x, y, alpha, beta, gacc);
  RVVLA_LAUNCHED("hcsr_spmv_kernel");
  return RVVLA_OK;
}

template <class V, class X, class SA, bool MIX>
int hcsr_spmv_impl(const rvvla_hcsr* A, X alpha, const X* x, X beta, X* y, cudaStream_t st) {
  using P = typename HTypes<V, X, SA, MIX>::P;
  int rc = hcsr_validate(A, x, y);
  if (rc) return rc;
  if (A->m == 0) return RVVLA_OK;
  if (A->b_m > INT32_MAX) return fail(RVVLA_ERR_TOO_LARGE, "hcsr: more than 2^31 - 1 block rows");
  const bool vec = ((uintptr_t)A->values % 16 == 0) && ((uintptr_t)A->col_idx % 16 == 0);
  const int64_t racc = std::min<int64_t>(A->R, A->m);
  const size_t smem_s = HLayout<SA, P>(racc).total;
  if (smem_s <= kHSmemMax) {
    return vec ? hcsr_launch<V, X, SA, MIX, true, false>(A, alpha, x, beta, y, nullptr, smem_s, st)
               : hcsr_launch<V, X, SA, MIX, false, false>(A, alpha, x, beta, y, nullptr, smem_s, st);
  }
  // block rows too tall for shared memory: the accumulator is a global
  // scratch array (each CTA owns its slice)
  Scratch sc;
  RVVLA_CUDA(sc.alloc((size_t)A->m * sizeof(SA), st));
  const size_t smem_g = HLayout<SA, P>(0).total;
  return vec ? hcsr_launch<V, X, SA, MIX, true, true>(A, alpha, x, beta, y, sc.as<SA>(), smem_g, st)
             : hcsr_launch<V, X, SA, MIX, false, true>(A, alpha, x, beta, y, sc.as<SA>(), smem_g, st);
}

}  // namespace
}  // namespace rvvla

using namespace rvvla;

extern "C" {

int rvvla_hcsr_spmv_f64(const rvvla_hcsr* A, double alpha, const double* x, double beta, double* y, void* stream) {
  return hcsr_spmv_impl<double, double, double, false>(A, alpha, x, beta, y, as_stream(stream));
}

int rvvla_hcsr_spmv_f32(const rvvla_hcsr* A, float alpha, const float* x, float beta, float* y, void* stream) {
  return hcsr_spmv_impl<float, float, float, false>(A, alpha, x, beta, y, as_stream(stream));
}

int rvvla_hcsr_spmv_mixed(const rvvla_hcsr* A, int val_type, float alpha, const float* x, float beta, float* y,
                          void* stream) {
  if (val_type == RVVLA_F32)
    return hcsr_spmv_impl<float, float, double, true>(A, alpha, x, beta, y, as_stream(stream));
  if (val_type == RVVLA_BF16)
    return hcsr_spmv_impl<__nv_bfloat16, float, double, true>(A, alpha, x, beta, y, as_stream(stream));
  return fail(RVVLA_ERR_INVALID_ARG, "hcsr_spmv_mixed: val_type must be RVVLA_F32 or RVVLA_BF16");
}

}  // extern "C"
