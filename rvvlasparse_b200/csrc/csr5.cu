// csr5.cu — spMtxCSR5 on sm_100a: GPU builder and y = alpha*A*x + beta*y.
//
// Layout (include/CSR5.h:57-112 of the reference; decode in
// src/rvv/spmv_mtx_csr5.cpp:85-296): tile t < p-1 holds nonzeros
// [t*w*s, (t+1)*w*s) stored transposed (CSR element tile_start + l*sigma + i
// at tile_start + i*omega + l); per lane, tile_desc_len descriptor dwords:
// y_offset (bit_y_offset bits), seg_offset (bit_seg_offset bits), then one
// row-start flag per step, MSB first; tile_pointer[t] = row of the tile's
// first element, bit 31 = the tile uses tile_empty_offset; the tail (from
// (p-1)*w*s) stays in CSR order.  The reference ships no builder (asCSR5 is
// declared, include/CSR5.h:61-65, never defined); this builder produces the
// layout the reference kernel decodes, bit-exact with the oracle's builder.
//
// SpMV mapping: omega = 32 = one warp; each warp walks a contiguous range of
// tiles (a CPU thread's chunk in :138-139).  Per tile every lane loads its
// sigma steps with coalesced 32-wide loads (values/columns L2 evict-first, x
// evict-last), then runs the reference's per-lane segment logic (green/red
// segments, :222-244) and replaces its slide-up scan plus gather-difference
// (:252-266) with a reverse segmented warp scan (same sums, no
// cancellation).  The row that crosses a tile boundary stays in a register
// carry (fp64 for the mixed form) until it ends, so every row is written once
// with alpha/beta; only rows that cross a WARP boundary go through the
// calibrator (:318-335), merged in warp order by a second kernel.  The tail
// rows use a third kernel (:337-365).  No float atomics: results are
// bitwise reproducible.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>

#include "rvvla_internal.cuh"
#include "scan.cuh"
#include "tma.cuh"

namespace rvvla {
namespace {

constexpr uint32_t kSign = 0x80000000u;
constexpr uint32_t kNoSign = 0x7FFFFFFFu;

int bits_for(int64_t v) {
  int r = 0;
  while (v) { r++; v >>= 1; }
  return r;
}

// ---------------------------------------------------------------- builder
__device__ __forceinline__ int64_t row_of(const int* Rst, int64_t m, int64_t e) {
  // largest r in [0, m] with Rst[r] <= e
  int64_t lo = 0, hi = m + 1;
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (Rst[mid] <= e) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void csr5_tileptr_kernel(int64_t p, int64_t ws, int64_t m, int64_t nnz, const int* __restrict__ Rst,
                                    uint32_t* __restrict__ tile_ptr) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t > p) return;
  tile_ptr[t] = (uint32_t)row_of(Rst, m, min(t * ws, nnz));
}

__global__ void csr5_startmark_kernel(int64_t m, const int* __restrict__ Rst, uint8_t* __restrict__ flag,
                                      int* __restrict__ srow, int* __restrict__ any_empty) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  const int a = Rst[r], b = Rst[r + 1];
  if (b > a) {
    flag[a] = 1;
    srow[a] = (int)r;
  } else {
    atomicOr(any_empty, 1);
  }
}

// One warp per full tile: descriptor dwords, empty-row flag, row-start count.
template <bool FILL>
__global__ void csr5_desc_kernel(int64_t nfull, int omega, int sigma, int by, int bsg, int tdl,
                                 const uint8_t* __restrict__ flag, const int* __restrict__ srow,
                                 uint32_t* __restrict__ tile_ptr, uint32_t* __restrict__ desc,
                                 int64_t* __restrict__ rs_count, const int64_t* __restrict__ eo_ptr,
                                 uint32_t* __restrict__ eo) {
  const int64_t t = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (t >= nfull) return;
  if (FILL && rs_count[t] == 0) return;  // only flagged tiles own map entries
  const int64_t ws = (int64_t)omega * sigma;
  const int64_t s0 = t * ws;
  const uint32_t first = tile_ptr[t] & kNoSign;
  const bool act = lane < omega;
  int cnt = 0;
  bool has = false;
  if (act) {
    for (int i = 0; i < sigma; ++i) {
      const int64_t e = (int64_t)lane * sigma + i;
      if (flag[s0 + e]) {
        has = true;
        if (e != 0) cnt++;
      }
    }
  }
  // exclusive scan of cnt over lanes -> y_offset
  int inc = cnt;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int o = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += o;
  }
  const int yoff = inc - cnt;
  const int total = __shfl_sync(0xffffffffu, inc, 31);
  const unsigned hasm = __ballot_sync(0xffffffffu, act && has);
  // seg_offset: following lanes without any row start
  const unsigned after = (lane < 31) ? (hasm & (~0u << (lane + 1))) : 0u;
  int seg = after ? (__ffs(after) - 1) - lane - 1 : (omega - 1 - lane);
  // identity of the empty-row map
  bool ident = true;
  if (act) {
    int k = yoff;
    for (int i = 0; i < sigma; ++i) {
      const int64_t e = (int64_t)lane * sigma + i;
      if (e != 0 && flag[s0 + e]) {
        const int row = srow[s0 + e];
        if (FILL) eo[eo_ptr[t] + k] = (uint32_t)(row - (int)first - 1);
        else if ((uint32_t)row != first + 1 + (uint32_t)k) ident = false;
        k++;
      }
    }
  }
  if (FILL) return;
  const bool flagged = __ballot_sync(0xffffffffu, !ident) != 0u;
  if (act) {
    uint32_t* d = desc + t * (int64_t)omega * tdl;
    const int flag0 = 32 - by - bsg;
    uint32_t w0 = ((uint32_t)yoff << (32 - by)) | ((uint32_t)seg << (32 - by - bsg));
    for (int i = 0; i < sigma && i < flag0; ++i)
      if (flag[s0 + (int64_t)lane * sigma + i]) w0 |= 1u << (31 - by - bsg - i);
    d[lane] = w0;
    for (int dw = 1; dw < tdl; ++dw) {
      uint32_t w = 0;
      for (int b = 0; b < 32; ++b) {
        const int i = flag0 + (dw - 1) * 32 + b;
        if (i < sigma && flag[s0 + (int64_t)lane * sigma + i]) w |= 1u << (31 - b);
      }
      d[(int64_t)dw * omega + lane] = w;
    }
  }
  if (lane == 0) {
    rs_count[t] = flagged ? total : 0;
    if (flagged) tile_ptr[t] |= kSign;
  }
}

// Transposed copy of the full tiles, straight copy of the tail.
template <int VB>
__global__ void csr5_copy_kernel(int64_t nnz, int64_t nfull, int omega, int sigma, const int* __restrict__ Col,
                                 const uint8_t* __restrict__ Val, uint32_t* __restrict__ col,
                                 uint8_t* __restrict__ val) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // destination index
  if (k >= nnz) return;
  const int64_t ws = (int64_t)omega * sigma;
  int64_t src = k;
  const int64_t t = k / ws;
  if (t < nfull) {
    const int64_t r = k - t * ws;
    const int64_t i = r / omega, l = r % omega;
    src = t * ws + l * sigma + i;
  }
  col[k] = (uint32_t)Col[src];
#pragma unroll
  for (int q = 0; q < VB; ++q) val[k * VB + q] = Val[src * VB + q];
}

__global__ void csr5_shift_kernel(int64_t n, const int64_t* __restrict__ in, uint32_t* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (uint32_t)in[i];
}

// ---------------------------------------------------------------- SpMV
__device__ __forceinline__ void cadd(double& a, double b) { a += b; }
__device__ __forceinline__ void cadd(float& a, float b) { a += b; }

template <class V, class X, class Ac, class CT>
struct LaneOps;
template <>
struct LaneOps<double, double, double, double> {
  __device__ static double prod(double v, double x) { return v * x; }
  __device__ static void add(double& a, double p) { a += p; }
  __device__ static double fin(double a) { return a; }
};
template <>
struct LaneOps<float, float, float, float> {
  __device__ static float prod(float v, float x) { return v * x; }
  __device__ static void add(float& a, float p) { a += p; }
  __device__ static float fin(float a) { return a; }
};
template <class V>
struct LaneOps<V, float, CompF32, double> {
  __device__ static float prod(V v, float x) { return to_f32(v) * x; }
  __device__ static void add(CompF32& a, float p) { a.add(p); }
  __device__ static double fin(const CompF32& a) { return (double)a.s + (double)a.c; }
};

template <class CT>
__device__ __forceinline__ CT shfl_down_ct(CT v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }

template <class X, class CT>
__device__ __forceinline__ void write_first(X* y, int64_t r, CT v, X alpha, X beta) {
  const X o = alpha * (X)v;
  y[r] = (beta == X(0)) ? o : o + beta * y[r];
}

constexpr int bits_ce(int v) { return v ? 1 + bits_ce(v >> 1) : 0; }

// Staging of a tile's values, columns and descriptor: straight into
// registers; through a per-warp shared-memory ring filled by bulk copies; or
// into registers one tile ahead (the next tile's loads overlap this tile's
// gathers and reduction, at about twice the registers).
constexpr int kC5Regs = 0, kC5Tma = 1, kC5Pipe = 2;

// Shared-memory pipeline geometry of the bulk-copy kernel: per warp, STAGES
// tiles of values + columns + descriptors (about 12 KB in flight per warp).
constexpr int kC5Warps = 4;
template <class V, int SIGMA>
struct C5Cfg {
  static constexpr int WS = 32 * SIGMA;
  static constexpr int TDL = (bits_ce(32 * SIGMA) + 6 + SIGMA + 31) / 32;
  static constexpr int VAL_B = WS * (int)sizeof(V);
  static constexpr int COL_B = WS * 4;
  static constexpr int DESC_B = 128 * TDL;
  static constexpr int STAGE_B = VAL_B + COL_B + DESC_B;
  static constexpr int STAGES = (12800 / STAGE_B) > 2 ? (12800 / STAGE_B) : 2;
  static constexpr int SMEM = kC5Warps * (STAGES * STAGE_B + STAGES * 8);
};

// One warp per contiguous tile range; omega == 32.  Lane 0 of each warp
// streams its tiles into a private STAGES-deep shared-memory ring with 1-D
// bulk copies (values, columns, descriptors; L2 evict-first) and mbarrier
// transaction counts; the warp gathers x for all SIGMA steps from registers
// while later tiles are in flight.
template <class V, class X, class Ac, class CT, int SIGMA, int MODE>
__global__ void __launch_bounds__(kC5Warps * 32)
csr5_spmv_kernel(int64_t nfull, int tiles_per_warp, const uint32_t* __restrict__ colidx,
                 const V* __restrict__ vals, const uint32_t* __restrict__ tile_ptr,
                 const uint32_t* __restrict__ desc, const uint32_t* __restrict__ eo_ptr,
                 const uint32_t* __restrict__ eo, const X* __restrict__ x, X* __restrict__ y, X alpha, X beta,
                 CT* __restrict__ cal, int* __restrict__ cal_row, int* __restrict__ status) {
  using Ops = LaneOps<V, X, Ac, CT>;
  using Cfg = C5Cfg<V, SIGMA>;
  // omega = 32 fixes the descriptor layout: bit_y_offset = bits(32*sigma),
  // bit_seg_offset = bits(32) = 6, so every flag position is a constant
  constexpr int S = Cfg::STAGES, TDL = Cfg::TDL;
  constexpr int BY = bits_ce(32 * SIGMA), BS = 6, FLAG0 = 32 - BY - BS;
  extern __shared__ __align__(128) unsigned char smem[];
  const int wid = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  unsigned char* wbuf = smem + wid * (S * Cfg::STAGE_B);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kC5Warps * S * Cfg::STAGE_B) + wid * S;
  const int64_t warp = (int64_t)blockIdx.x * kC5Warps + wid;
  const int64_t t0 = warp * tiles_per_warp;
  if (t0 >= nfull) return;
  const int64_t t1 = min(nfull, t0 + tiles_per_warp);
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  auto issue = [&](int64_t t, int s) {
    unsigned char* st = wbuf + s * Cfg::STAGE_B;
    mbar_expect_tx(&bars[s], (uint32_t)Cfg::STAGE_B);
    bulk_g2s(st, vals + t * Cfg::WS, Cfg::VAL_B, &bars[s], pf);
    bulk_g2s(st + Cfg::VAL_B, colidx + t * Cfg::WS, Cfg::COL_B, &bars[s], pf);
    bulk_g2s(st + Cfg::VAL_B + Cfg::COL_B, desc + t * 32 * TDL, Cfg::DESC_B, &bars[s], pf);
  };
  constexpr bool TMA = MODE == kC5Tma;
  if constexpr (TMA) {
    if (lane == 0) {
      for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
      fence_mbar_init();
    }
    __syncwarp();
    if (lane == 0)
      for (int s = 0; s < S && t0 + s < t1; ++s) issue(t0 + s, s);
  }
  int64_t crow = -1;
  CT cval = 0;
  bool cfirst = true;  // false: the row started before this warp -> calibrator
  {
    const uint32_t d0 = __shfl_sync(0xffffffffu, desc[t0 * 32 * TDL + lane], 0);
    if (!((d0 >> (31 - BY - BS)) & 1u)) {
      crow = tile_ptr[t0] & kNoSign;
      cfirst = false;
    }
  }
  int64_t calrow = -1;
  CT calv = 0;
  auto flush = [&]() {
    if (crow >= 0) {
      if (cfirst) {
        if (lane == 0) write_first(y, crow, cval, alpha, beta);
      } else {
        calrow = crow;
        calv = cval;
      }
    }
    crow = -1;
    cval = 0;
    cfirst = true;
  };
  using PT = decltype(Ops::prod(V(), X()));
  // register variant: the columns, values and descriptor of tile t+1 are
  // loaded before tile t gathers x, so the stream loads of the next tile are
  // in flight during this tile's gathers and reduction
  uint32_t cn[SIGMA];
  V vn[SIGMA];
  uint32_t dwn[TDL];
  auto load_tile = [&](int64_t t) {
    const int64_t base = t * (int64_t)Cfg::WS;
#pragma unroll
    for (int i = 0; i < SIGMA; ++i) cn[i] = ld_stream(colidx + base + i * 32 + lane, pf);
#pragma unroll
    for (int i = 0; i < SIGMA; ++i) vn[i] = ld_stream(vals + base + i * 32 + lane, pf);
#pragma unroll
    for (int d = 0; d < TDL; ++d) dwn[d] = ld_stream(desc + t * 32 * TDL + d * 32 + lane, pf);
  };
  if constexpr (MODE == kC5Pipe) load_tile(t0);
  for (int64_t t = t0; t < t1; ++t) {
    const int64_t it = t - t0;
    const int s = (int)(it % S);
    PT prod[SIGMA];
    uint32_t dw[TDL];
    if constexpr (TMA) {
      if (!mbar_wait(&bars[s], (uint32_t)((it / S) & 1))) {
        // a copy never completed: record it, drain what is in flight, leave
        if (lane == 0) {
          atomicOr(status, RVVLA_DEV_ERR_TIMEOUT);
          for (int64_t u = t + 1; u < t1 && u < t + S; ++u)
            mbar_wait(&bars[(u - t0) % S], (uint32_t)(((u - t0) / S) & 1));
        }
        __syncwarp();
        return;
      }
      const unsigned char* st = wbuf + s * Cfg::STAGE_B;
      const V* sv = reinterpret_cast<const V*>(st);
      const uint32_t* sc = reinterpret_cast<const uint32_t*>(st + Cfg::VAL_B);
      const uint32_t* sd = reinterpret_cast<const uint32_t*>(st + Cfg::VAL_B + Cfg::COL_B);
      uint32_t c[SIGMA];
      V v[SIGMA];
#pragma unroll
      for (int i = 0; i < SIGMA; ++i) c[i] = sc[i * 32 + lane];
#pragma unroll
      for (int i = 0; i < SIGMA; ++i) v[i] = sv[i * 32 + lane];
#pragma unroll
      for (int d = 0; d < TDL; ++d) dw[d] = sd[d * 32 + lane];
      // the warp is done with this stage: refill it with tile t+S
      __syncwarp();
      if (lane == 0 && t + S < t1) {
        fence_proxy_async();
        issue(t + S, s);
      }
#pragma unroll
      for (int i = 0; i < SIGMA; ++i) prod[i] = Ops::prod(v[i], ld_keep(x + c[i], pl));
    } else {
      if constexpr (MODE == kC5Regs) load_tile(t);
      uint32_t c[SIGMA];
      V v[SIGMA];
#pragma unroll
      for (int i = 0; i < SIGMA; ++i) c[i] = cn[i];
#pragma unroll
      for (int i = 0; i < SIGMA; ++i) v[i] = vn[i];
#pragma unroll
      for (int d = 0; d < TDL; ++d) dw[d] = dwn[d];
      if constexpr (MODE == kC5Pipe)
        if (t + 1 < t1) load_tile(t + 1);
#pragma unroll
      for (int i = 0; i < SIGMA; ++i) prod[i] = Ops::prod(v[i], ld_keep(x + c[i], pl));
    }
    const uint32_t tp = tile_ptr[t];
    const bool empty = (tp >> 31) & 1u;
    const int64_t first = tp & kNoSign;
    const uint32_t optr = empty ? eo_ptr[t] : 0u;
    uint32_t yoff = dw[0] >> (32 - BY);
    const uint32_t f0 = dw[0] << (BY + BS);  // step i (< FLAG0) at bit 31-i
    bool lb = (f0 >> 31) & 1u;
    const bool step0_start = lb;
    if (lane == 0) lb = true;
    const bool start = !lb;
    bool incol = lb && lane != 0;
    Ac sum = Ac(), fsum = Ac();
    Ops::add(sum, prod[0]);
#pragma unroll
    for (int i = 1; i < SIGMA; ++i) {
      const bool flag = (i < FLAG0) ? ((f0 >> (31 - i)) & 1u)
                                    : ((dw[(i - FLAG0) / 32 + 1] >> (31 - (i - FLAG0) % 32)) & 1u);
      if (flag) {
        if (incol) {  // a full row that started in this lane
          const uint32_t k = empty ? eo[optr + yoff] : yoff;
          write_first(y, first + 1 + k, (CT)Ops::fin(sum), alpha, beta);
          yoff++;
        } else {
          fsum = sum;
        }
        sum = Ac();
        incol = true;
      }
      Ops::add(sum, prod[i]);
    }
    // lead: the part of this lane that belongs to the previous lane's row
    const CT lead = start ? (incol ? (CT)Ops::fin(fsum) : (CT)Ops::fin(sum)) : CT(0);
    const bool has_start = step0_start || incol;
    const unsigned stops = __ballot_sync(0xffffffffu, has_start);
    const unsigned ge = stops & (~0u << lane);
    const int e = ge ? __ffs(ge) - 1 : 31;
    CT T = lead;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const CT o = shfl_down_ct(T, d);
      if (lane + d <= e) T += o;
    }
    CT Tn = shfl_down_ct(T, 1);
    if (lane == 31) Tn = 0;
    const CT lastv = (CT)Ops::fin(sum) + Tn;
    const bool incol0 = __shfl_sync(0xffffffffu, incol, 0);
    const CT fs0 = __shfl_sync(0xffffffffu, (CT)Ops::fin(fsum), 0);
    const CT add = incol0 ? fs0 : __shfl_sync(0xffffffffu, lastv, 0);
    const unsigned incm = __ballot_sync(0xffffffffu, incol);
    if (crow >= 0 && crow != first) flush();
    if (crow == first) cadd(cval, add);
    else {
      crow = first;
      cval = add;
      cfirst = true;
    }
    if (incm) {
      flush();  // the tile's first row ends in this tile
      const int lstar = 31 - __clz(incm);
      if (incol && lane != lstar) {
        const uint32_t k = empty ? eo[optr + yoff] : yoff;
        write_first(y, first + 1 + k, lastv, alpha, beta);
      }
      const uint32_t ks = __shfl_sync(0xffffffffu, empty ? (incol ? eo[optr + yoff] : 0u) : yoff, lstar);
      crow = first + 1 + ks;
      cval = __shfl_sync(0xffffffffu, lastv, lstar);
      cfirst = true;
    }
  }
  flush();
  if (lane == 0) {
    cal_row[warp] = (int)calrow;
    cal[warp] = calv;
  }
}

// Generic-sigma variant (runtime loop) for sigma values without a template.
template <class V, class X, class Ac, class CT>
__global__ void __launch_bounds__(256)
csr5_spmv_generic_kernel(int64_t nfull, int tiles_per_warp, int sigma, int by, int bsg, int tdl,
                         const uint32_t* __restrict__ colidx, const V* __restrict__ vals,
                         const uint32_t* __restrict__ tile_ptr, const uint32_t* __restrict__ desc,
                         const uint32_t* __restrict__ eo_ptr, const uint32_t* __restrict__ eo,
                         const X* __restrict__ x, X* __restrict__ y, X alpha, X beta, CT* __restrict__ cal,
                         int* __restrict__ cal_row) {
  using Ops = LaneOps<V, X, Ac, CT>;
  const int64_t warp = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const int64_t t0 = warp * tiles_per_warp;
  if (t0 >= nfull) return;
  const int64_t t1 = min(nfull, t0 + tiles_per_warp);
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  const int flag0 = 32 - by - bsg;
  const int bit0 = 31 - by - bsg;
  int64_t crow = -1;
  CT cval = 0;
  bool cfirst = true;
  {
    const uint32_t d0 = __shfl_sync(0xffffffffu, desc[t0 * 32 * tdl + lane], 0);
    if (!((d0 >> bit0) & 1u)) {
      crow = tile_ptr[t0] & kNoSign;
      cfirst = false;
    }
  }
  int64_t calrow = -1;
  CT calv = 0;
  auto flush = [&]() {
    if (crow >= 0) {
      if (cfirst) {
        if (lane == 0) write_first(y, crow, cval, alpha, beta);
      } else {
        calrow = crow;
        calv = cval;
      }
    }
    crow = -1;
    cval = 0;
    cfirst = true;
  };
  for (int64_t t = t0; t < t1; ++t) {
    const int64_t base = t * (32 * (int64_t)sigma);
    const uint32_t* dt = desc + t * 32 * tdl;
    uint32_t dw = dt[lane];
    const uint32_t tp = tile_ptr[t];
    const bool empty = (tp >> 31) & 1u;
    const int64_t first = tp & kNoSign;
    const uint32_t optr = empty ? eo_ptr[t] : 0u;
    uint32_t yoff = dw >> (32 - by);
    uint32_t cur = dw << (by + bsg);
    bool lb = (cur >> 31) & 1u;
    const bool step0_start = lb;
    if (lane == 0) lb = true;
    const bool start = !lb;
    bool incol = lb && lane != 0;
    Ac sum = Ac(), fsum = Ac();
    Ops::add(sum, Ops::prod(ld_stream(vals + base + lane, pf), ld_keep(x + ld_stream(colidx + base + lane, pf), pl)));
    int ly = 0;
    for (int i = 1; i < sigma; ++i) {
      const uint32_t ci = ld_stream(colidx + base + (int64_t)i * 32 + lane, pf);
      const V vi = ld_stream(vals + base + (int64_t)i * 32 + lane, pf);
      const int norm_i = i - flag0;
      if (norm_i >= 0 && (norm_i % 32) == 0) {
        ly++;
        cur = dt[ly * 32 + lane];
      }
      const int ni = (ly == 0) ? i : (norm_i % 32);
      if ((cur >> (31 - ni)) & 1u) {
        if (incol) {
          const uint32_t k = empty ? eo[optr + yoff] : yoff;
          write_first(y, first + 1 + k, (CT)Ops::fin(sum), alpha, beta);
          yoff++;
        } else {
          fsum = sum;
        }
        sum = Ac();
        incol = true;
      }
      Ops::add(sum, Ops::prod(vi, ld_keep(x + ci, pl)));
    }
    const CT lead = start ? (incol ? (CT)Ops::fin(fsum) : (CT)Ops::fin(sum)) : CT(0);
    const bool has_start = step0_start || incol;
    const unsigned stops = __ballot_sync(0xffffffffu, has_start);
    const unsigned ge = stops & (~0u << lane);
    const int e = ge ? __ffs(ge) - 1 : 31;
    CT T = lead;
    for (int d = 1; d < 32; d <<= 1) {
      const CT o = shfl_down_ct(T, d);
      if (lane + d <= e) T += o;
    }
    CT Tn = shfl_down_ct(T, 1);
    if (lane == 31) Tn = 0;
    const CT lastv = (CT)Ops::fin(sum) + Tn;
    const bool incol0 = __shfl_sync(0xffffffffu, incol, 0);
    const CT fs0 = __shfl_sync(0xffffffffu, (CT)Ops::fin(fsum), 0);
    const CT add = incol0 ? fs0 : __shfl_sync(0xffffffffu, lastv, 0);
    const unsigned incm = __ballot_sync(0xffffffffu, incol);
    if (crow >= 0 && crow != first) flush();
    if (crow == first) cadd(cval, add);
    else {
      crow = first;
      cval = add;
      cfirst = true;
    }
    if (incm) {
      flush();
      const int lstar = 31 - __clz(incm);
      if (incol && lane != lstar) {
        const uint32_t k = empty ? eo[optr + yoff] : yoff;
        write_first(y, first + 1 + k, lastv, alpha, beta);
      }
      const uint32_t ks = __shfl_sync(0xffffffffu, empty ? (incol ? eo[optr + yoff] : 0u) : yoff, lstar);
      crow = first + 1 + ks;
      cval = __shfl_sync(0xffffffffu, lastv, lstar);
      cfirst = true;
    }
  }
  flush();
  if (lane == 0) {
    cal_row[warp] = (int)calrow;
    cal[warp] = calv;
  }
}

// Calibrator merge in warp order (:318-335): a run of warps continuing one
// row is summed first, then added once.
template <class X, class CT>
__global__ void csr5_calibrate_kernel(int64_t nwarps, const int* __restrict__ cal_row, const CT* __restrict__ cal,
                                      X* __restrict__ y, X alpha) {
  const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nwarps) return;
  const int r = cal_row[w];
  if (r < 0) return;
  if (w > 0 && cal_row[w - 1] == r) return;
  CT s = cal[w];
  for (int64_t u = w + 1; u < nwarps && cal_row[u] == r; ++u) s += cal[u];
  y[r] += alpha * (X)s;
}

// Tail rows (:337-365): one warp per row from tail_tile_start; the first
// tail row continues a row begun in the last full tile unless it starts
// exactly at the tail.
template <class V, class X, class Ac, class CT>
__global__ void csr5_tail_kernel(int64_t m, int64_t tail_row, int64_t tail_start, const int* __restrict__ Rst,
                                 const uint32_t* __restrict__ colidx, const V* __restrict__ vals,
                                 const X* __restrict__ x, X* __restrict__ y, X alpha, X beta) {
  using Ops = LaneOps<V, X, Ac, CT>;
  const int64_t r = tail_row + (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= m) return;
  const int64_t kb = (r == tail_row) ? tail_start : Rst[r];
  const int64_t ke = Rst[r + 1];
  Ac s = Ac();
  for (int64_t k = kb + lane; k < ke; k += 32) Ops::add(s, Ops::prod(vals[k], x[colidx[k]]));
  CT v = (CT)Ops::fin(s);
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  if (lane == 0) {
    const bool cont = (r == tail_row) && (Rst[r] < tail_start);
    if (cont) y[r] += alpha * (X)v;
    else write_first(y, r, v, alpha, beta);
  }
}

template <class X>
__global__ void scale_kernel(int64_t m, X* __restrict__ y, X beta) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) y[i] = (beta == X(0)) ? X(0) : beta * y[i];
}

// Staging variant of the templated kernel (a tuning knob read once:
// RVVLA_CSR5_STAGING=regs|tma|pipe).  Default: registers, which measured
// faster on B200 than the shared-memory ring (up to 28 resident warps per SM
// against 16).
int csr5_staging() {
  static const int mode = [] {
    const char* e = std::getenv("RVVLA_CSR5_STAGING");
    const std::string v = e ? e : "";
    return v == "tma" ? kC5Tma : v == "pipe" ? kC5Pipe : kC5Regs;
  }();
  return mode;
}

int csr5_validate(const rvvla_csr5* A, const void* x, const void* y) {
  if (!A) return fail(RVVLA_ERR_INVALID_ARG, "csr5: null descriptor");
  if (A->m < 0 || A->n < 0 || A->nnz < 0 || A->p < 1 || A->sigma <= 0 || A->omega <= 0)
    return fail(RVVLA_ERR_INVALID_ARG, "csr5: bad sizes");
  if (A->omega != 32) return fail(RVVLA_ERR_UNSUPPORTED, "csr5: the sm_100a kernel needs omega == 32 (one warp)");
  if (A->bit_y_offset + A->bit_seg_offset >= 32 || A->tile_desc_len < 1)
    return fail(RVVLA_ERR_FORMAT, "csr5: bad descriptor bit widths");
  if ((int64_t)(A->p - 1) * A->omega * A->sigma > A->nnz) return fail(RVVLA_ERR_FORMAT, "csr5: p inconsistent with nnz");
  if (A->m > 0 && (!A->csr_row_pointer || !A->tile_pointer || !y)) return fail(RVVLA_ERR_INVALID_ARG, "csr5: null array");
  if (A->nnz > 0 && (!A->csr_column_index || !A->csr_value || !x)) return fail(RVVLA_ERR_INVALID_ARG, "csr5: null array");
  if (A->p > 1 && !A->tile_descriptor) return fail(RVVLA_ERR_INVALID_ARG, "csr5: null descriptor array");
  return RVVLA_OK;
}

// Warps per SM the compiled (sigma, staging) kernel keeps resident, capped at
// 48: the SpMV launches one wave of exactly that many warps per SM (each warp
// gets an equal share of tiles), so no partial second wave trails the grid.
template <class V, class X, class Ac, class CT>
int c5_resident_warps(int sigma, int mode) {
  // per device (GPUs of one machine may differ), written once per entry;
  // concurrent first calls compute the same value
  constexpr int kDev = 16;
  static std::atomic<int> cache[kDev][4][3];  // static storage: zero-initialised
  const int si = sigma / 8 - 1;
  if (si < 0 || si > 3 || sigma % 8 || mode < 0 || mode > 2) return 48;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDev) {
    cudaGetLastError();
    dev = -1;
  }
  int c = dev >= 0 ? cache[dev][si][mode].load(std::memory_order_relaxed) : 0;
  if (c == 0) {
    int blocks = 0;
    cudaError_t e = cudaErrorInvalidValue;
    switch (sigma) {
#define C5_OCC(S)                                                                                             \
  case S:                                                                                                     \
    e = mode == kC5Tma                                                                                        \
            ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, csr5_spmv_kernel<V, X, Ac, CT, S, kC5Tma>, \
                                                            kC5Warps * 32, C5Cfg<V, S>::SMEM)                 \
        : mode == kC5Pipe                                                                                     \
            ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, csr5_spmv_kernel<V, X, Ac, CT, S, kC5Pipe>, \
                                                            kC5Warps * 32, 0)                                 \
            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, csr5_spmv_kernel<V, X, Ac, CT, S, kC5Regs>, \
                                                            kC5Warps * 32, 0);                                \
    break;
      C5_OCC(8)
      C5_OCC(16)
      C5_OCC(24)
      C5_OCC(32)
#undef C5_OCC
    }
    c = (e == cudaSuccess && blocks > 0) ? std::min(48, blocks * kC5Warps) : 48;
    if (e != cudaSuccess) cudaGetLastError();
    if (dev >= 0) cache[dev][si][mode].store(c, std::memory_order_relaxed);
  }
  return c;
}

template <class V, class X, class Ac, class CT>
int csr5_spmv_impl(const rvvla_csr5* A, X alpha, const X* x, X beta, X* y, cudaStream_t st, CT* cal_buf,
                   int* cal_row_buf, int64_t cal_cap, int* status_word, bool regs_only) {
  int rc = csr5_validate(A, x, y);
  if (rc) return rc;
  if (A->m == 0) return RVVLA_OK;
  X beta_eff = beta;
  if (!A->no_empty_rows) {
    scale_kernel<X><<<(unsigned)((A->m + 255) / 256), 256, 0, st>>>(A->m, y, beta);
    RVVLA_LAUNCHED("csr5 scale_kernel");
    beta_eff = X(1);
  }
  const int64_t nfull = A->p - 1;
  if (nfull > 0) {
    // bulk copies need 16-byte aligned sources; other layouts take the
    // register-only kernel
    const bool aligned = ((uintptr_t)A->csr_value % 16 == 0) && ((uintptr_t)A->csr_column_index % 16 == 0) &&
                         ((uintptr_t)A->tile_descriptor % 16 == 0);
    // regs_only: the register-staged kernel whatever the staging knob says
    // (no TMA ring, no doubled register set)
    const int mode = regs_only ? kC5Regs : csr5_staging();
    const int per_sm = aligned ? c5_resident_warps<V, X, Ac, CT>(A->sigma, mode) : 48;
    const int64_t want_warps = (int64_t)sm_count() * per_sm;
    int tpw = (int)std::max<int64_t>(1, (nfull + want_warps - 1) / want_warps);
    const int64_t nwarps = (nfull + tpw - 1) / tpw;
    Scratch sc;
    CT* cal = cal_buf;
    int* cal_row = cal_row_buf;
    if (!cal) {
      RVVLA_CUDA(sc.alloc((size_t)nwarps * (sizeof(CT) + sizeof(int)) + 256, st));
      cal = sc.as<CT>();
      cal_row = reinterpret_cast<int*>(sc.as<char>() + ((size_t)nwarps * sizeof(CT) + 255) / 256 * 256);
    } else if (nwarps > cal_cap) {
      return fail(RVVLA_ERR_TOO_LARGE, "csr5: calibrator capacity too small for this matrix");
    }
    const unsigned blocks = (unsigned)((nwarps + 7) / 8);
    const uint32_t* eo_ptr = A->tile_empty_offset_pointer;
    const uint32_t* eo = A->tile_empty_offset;
    const V* vals = (const V*)A->csr_value;
    int* status = status_word ? status_word : device_status_word();
    if (!status) return fail(RVVLA_ERR_CUDA, "csr5: no device status word");
    switch (aligned ? A->sigma : -1) {
#define CSR5_CASE(S)                                                                                         \
  case S: {                                                                                                  \
    auto k_ = csr5_spmv_kernel<V, X, Ac, CT, S, kC5Regs>;                                                    \
    if (mode == kC5Tma) k_ = csr5_spmv_kernel<V, X, Ac, CT, S, kC5Tma>;                                      \
    if (mode == kC5Pipe) k_ = csr5_spmv_kernel<V, X, Ac, CT, S, kC5Pipe>;                                    \
    const int smem_ = mode == kC5Tma ? C5Cfg<V, S>::SMEM : 0;                                                \
    if (A->tile_desc_len != C5Cfg<V, S>::TDL || A->bit_y_offset != bits_ce(32 * S) || A->bit_seg_offset != 6)  \
      return fail(RVVLA_ERR_FORMAT, "csr5: descriptor widths do not match omega=32, sigma");                 \
    if (smem_ > 48 * 1024)                                                                                   \
      RVVLA_CUDA(cudaFuncSetAttribute(k_, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_));              \
    const int64_t nw_ = nwarps;                                                                              \
    k_<<<(unsigned)((nw_ + kC5Warps - 1) / kC5Warps), kC5Warps * 32, smem_, st>>>(                           \
        nfull, tpw, A->csr_column_index, vals, A->tile_pointer,                                              \
        A->tile_descriptor, eo_ptr, eo, x, y, alpha, beta_eff, cal, cal_row, status);                        \
    break;                                                                                                   \
  }
      CSR5_CASE(8)
      CSR5_CASE(16)
      CSR5_CASE(24)
      CSR5_CASE(32)
#undef CSR5_CASE
      default:
        csr5_spmv_generic_kernel<V, X, Ac, CT><<<blocks, 256, 0, st>>>(
            nfull, tpw, A->sigma, A->bit_y_offset, A->bit_seg_offset, A->tile_desc_len, A->csr_column_index, vals,
            A->tile_pointer, A->tile_descriptor, eo_ptr, eo, x, y, alpha, beta_eff, cal, cal_row);
    }
    RVVLA_LAUNCHED("csr5_spmv_kernel");
    csr5_calibrate_kernel<X, CT><<<(unsigned)((nwarps + 255) / 256), 256, 0, st>>>(nwarps, cal_row, cal, y, alpha);
    RVVLA_LAUNCHED("csr5_calibrate_kernel");
  }
  if (A->tail_tile_start < A->m) {
    const int64_t rows = A->m - A->tail_tile_start;
    csr5_tail_kernel<V, X, Ac, CT><<<(unsigned)((rows + 7) / 8), 256, 0, st>>>(
        A->m, A->tail_tile_start, (int64_t)(A->p - 1) * A->omega * A->sigma, A->csr_row_pointer, A->csr_column_index,
        (const V*)A->csr_value, x, y, alpha, beta_eff);
    RVVLA_LAUNCHED("csr5_tail_kernel");
  }
  return RVVLA_OK;
}

}  // namespace

int csr5_build_impl(const rvvla_crs* src, int vb, int omega, int sigma, rvvla_csr5_owned* out, cudaStream_t st) {
  if (!src || !out) return fail(RVVLA_ERR_INVALID_ARG, "csr5_build: null argument");
  std::memset(out, 0, sizeof(*out));
  if (omega <= 0 || sigma <= 0) return fail(RVVLA_ERR_INVALID_ARG, "CSR5: omega and sigma must be positive");
  if (omega > 32) return fail(RVVLA_ERR_UNSUPPORTED, "CSR5: the GPU builder supports omega <= 32");
  if (vb != 8 && vb != 4 && vb != 2) return fail(RVVLA_ERR_INVALID_ARG, "csr5_build: val_bytes must be 8, 4 or 2");
  const int64_t m = src->m, n = src->n, nnz = src->nz, ws = (int64_t)omega * sigma;
  if (m < 0 || n < 0 || nnz < 0) return fail(RVVLA_ERR_INVALID_ARG, "csr5_build: bad sizes");
  if (m >= INT32_MAX || nnz >= INT32_MAX) return fail(RVVLA_ERR_TOO_LARGE, "csr5_build: m or nnz beyond int32");
  int64_t p = (nnz + ws - 1) / ws;
  if (p < 1) p = 1;
  const int by = bits_for(ws), bsg = bits_for(omega);
  if (by + bsg >= 32) return fail(RVVLA_ERR_INVALID_ARG, "CSR5: omega*sigma too large");
  const int tdl = (by + bsg + sigma + 31) / 32;
  const int64_t nfull = p - 1;
  rvvla_csr5& h = out->h;
  h.m = m; h.n = n; h.nnz = nnz; h.bit_y_offset = by; h.bit_seg_offset = bsg; h.tile_desc_len = tdl;
  h.p = (int32_t)p; h.omega = omega; h.sigma = sigma;
  RVVLA_CUDA(cudaMalloc(&out->csr_row_pointer, (size_t)(m + 1) * sizeof(int32_t)));
  RVVLA_CUDA(cudaMalloc(&out->csr_column_index, (size_t)std::max<int64_t>(nnz, 1) * sizeof(uint32_t)));
  RVVLA_CUDA(cudaMalloc(&out->csr_value, (size_t)std::max<int64_t>(nnz, 1) * vb));
  RVVLA_CUDA(cudaMalloc(&out->tile_pointer, (size_t)(p + 1) * sizeof(uint32_t)));
  RVVLA_CUDA(cudaMalloc(&out->tile_descriptor, (size_t)std::max<int64_t>(nfull * omega * tdl, 1) * sizeof(uint32_t)));
  RVVLA_CUDA(cudaMalloc(&out->tile_empty_offset_pointer, (size_t)p * sizeof(uint32_t)));
  RVVLA_CUDA(cudaMemcpyAsync(out->csr_row_pointer, src->Rst, (size_t)(m + 1) * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
  csr5_tileptr_kernel<<<(unsigned)((p + 1 + 255) / 256), 256, 0, st>>>(p, ws, m, nnz, src->Rst, out->tile_pointer);
  RVVLA_LAUNCHED("csr5_tileptr_kernel");
  Scratch s_flag, s_srow, s_cnt, s_eop, s_any;
  RVVLA_CUDA(s_flag.alloc((size_t)std::max<int64_t>(nnz, 1), st));
  RVVLA_CUDA(s_srow.alloc((size_t)std::max<int64_t>(nnz, 1) * sizeof(int), st));
  RVVLA_CUDA(s_cnt.alloc((size_t)(p + 1) * sizeof(int64_t), st));
  RVVLA_CUDA(s_eop.alloc((size_t)(p + 1) * sizeof(int64_t), st));
  RVVLA_CUDA(s_any.alloc(sizeof(int), st));
  RVVLA_CUDA(cudaMemsetAsync(s_flag.p, 0, (size_t)std::max<int64_t>(nnz, 1), st));
  RVVLA_CUDA(cudaMemsetAsync(s_any.p, 0, sizeof(int), st));
  RVVLA_CUDA(cudaMemsetAsync(s_cnt.p, 0, (size_t)(p + 1) * sizeof(int64_t), st));
  if (m > 0) {
    csr5_startmark_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(m, src->Rst, s_flag.as<uint8_t>(),
                                                                        s_srow.as<int>(), s_any.as<int>());
    RVVLA_LAUNCHED("csr5_startmark_kernel");
  }
  if (nfull > 0) {
    csr5_desc_kernel<false><<<(unsigned)((nfull + 7) / 8), 256, 0, st>>>(
        nfull, omega, sigma, by, bsg, tdl, s_flag.as<uint8_t>(), s_srow.as<int>(), out->tile_pointer,
        out->tile_descriptor, s_cnt.as<int64_t>(), nullptr, nullptr);
    RVVLA_LAUNCHED("csr5_desc_kernel");
  }
  int rc = exclusive_scan_i64(s_cnt.as<int64_t>(), s_eop.as<int64_t>(), p, st);
  if (rc) return rc;
  int64_t nofs = 0;
  int any_empty = 0;
  uint32_t tail_row = 0;
  RVVLA_CUDA(cudaMemcpyAsync(&nofs, s_eop.as<int64_t>() + p, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaMemcpyAsync(&any_empty, s_any.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaMemcpyAsync(&tail_row, out->tile_pointer + (p - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaStreamSynchronize(st));
  csr5_shift_kernel<<<(unsigned)((p + 255) / 256), 256, 0, st>>>(p, s_eop.as<int64_t>(), out->tile_empty_offset_pointer);
  RVVLA_LAUNCHED("csr5_shift_kernel");
  RVVLA_CUDA(cudaMalloc(&out->tile_empty_offset, (size_t)std::max<int64_t>(nofs, 1) * sizeof(uint32_t)));
  if (nofs > 0) {
    csr5_desc_kernel<true><<<(unsigned)((nfull + 7) / 8), 256, 0, st>>>(
        nfull, omega, sigma, by, bsg, tdl, s_flag.as<uint8_t>(), s_srow.as<int>(), out->tile_pointer,
        out->tile_descriptor, s_cnt.as<int64_t>(), s_eop.as<int64_t>(), out->tile_empty_offset);
    RVVLA_LAUNCHED("csr5_desc_kernel(fill)");
  }
  if (nnz > 0) {
    const unsigned blocks = (unsigned)((nnz + 255) / 256);
    if (vb == 8) csr5_copy_kernel<8><<<blocks, 256, 0, st>>>(nnz, nfull, omega, sigma, src->Col, (const uint8_t*)src->Val, out->csr_column_index, (uint8_t*)out->csr_value);
    else if (vb == 4) csr5_copy_kernel<4><<<blocks, 256, 0, st>>>(nnz, nfull, omega, sigma, src->Col, (const uint8_t*)src->Val, out->csr_column_index, (uint8_t*)out->csr_value);
    else csr5_copy_kernel<2><<<blocks, 256, 0, st>>>(nnz, nfull, omega, sigma, src->Col, (const uint8_t*)src->Val, out->csr_column_index, (uint8_t*)out->csr_value);
    RVVLA_LAUNCHED("csr5_copy_kernel");
  }
  h.num_offsets = (int32_t)nofs;
  h.tail_tile_start = (int32_t)(tail_row & kNoSign);
  h.no_empty_rows = any_empty ? 0 : 1;
  h.csr_row_pointer = out->csr_row_pointer;
  h.csr_column_index = out->csr_column_index;
  h.csr_value = out->csr_value;
  h.tile_pointer = out->tile_pointer;
  h.tile_descriptor = out->tile_descriptor;
  h.tile_empty_offset_pointer = out->tile_empty_offset_pointer;
  h.tile_empty_offset = out->tile_empty_offset;
  RVVLA_CUDA(cudaStreamSynchronize(st));
  return RVVLA_OK;
}

template <class V, class X, class Ac, class CT>
int csr5_spmv_dispatch(const rvvla_csr5* A, X alpha, const X* x, X beta, X* y, cudaStream_t st, CT* cal,
                       int* cal_row, int64_t cap, int* status_word, bool regs_only) {
  return csr5_spmv_impl<V, X, Ac, CT>(A, alpha, x, beta, y, st, cal, cal_row, cap, status_word, regs_only);
}

// Upper bound of the calibrator entries the SpMV of this matrix needs (one
// per warp; the launch uses at most 48 warps per SM).
int64_t csr5_calibrator_len(const rvvla_csr5* A) {
  const int64_t nfull = A->p - 1;
  if (nfull <= 0) return 0;
  const int64_t want = (int64_t)sm_count() * 48;
  const int64_t tpw = std::max<int64_t>(1, (nfull + want - 1) / want);
  return (nfull + tpw - 1) / tpw;
}

template int csr5_spmv_dispatch<double, double, double, double>(const rvvla_csr5*, double, const double*, double,
                                                                double*, cudaStream_t, double*, int*, int64_t,
                                                                int*, bool);
template int csr5_spmv_dispatch<float, float, float, float>(const rvvla_csr5*, float, const float*, float, float*,
                                                            cudaStream_t, float*, int*, int64_t, int*, bool);
template int csr5_spmv_dispatch<float, float, CompF32, double>(const rvvla_csr5*, float, const float*, float,
                                                               float*, cudaStream_t, double*, int*, int64_t, int*,
                                                               bool);
template int csr5_spmv_dispatch<__nv_bfloat16, float, CompF32, double>(const rvvla_csr5*, float, const float*,
                                                                       float, float*, cudaStream_t, double*, int*,
                                                                       int64_t, int*, bool);

}  // namespace rvvla

using namespace rvvla;

extern "C" {

int rvvla_csr5_build(const rvvla_crs* src, int val_bytes, int omega, int sigma, rvvla_csr5_owned* out,
                     void* stream) {
  int rc = csr5_build_impl(src, val_bytes, omega, sigma, out, as_stream(stream));
  if (rc && out) {
    std::string keep = rvvla_last_error();
    rvvla_csr5_free(out);
    set_error(keep);
  }
  return rc;
}

void rvvla_csr5_free(rvvla_csr5_owned* h) {
  if (!h) return;
  cudaFree(h->csr_row_pointer);
  cudaFree(h->csr_column_index);
  cudaFree(h->csr_value);
  cudaFree(h->tile_pointer);
  cudaFree(h->tile_descriptor);
  cudaFree(h->tile_empty_offset_pointer);
  cudaFree(h->tile_empty_offset);
  std::memset(h, 0, sizeof(*h));
}

int rvvla_csr5_spmv_f64(const rvvla_csr5* A, double alpha, const double* x, double beta, double* y, void* stream) {
  return csr5_spmv_dispatch<double, double, double, double>(A, alpha, x, beta, y, as_stream(stream), nullptr,
                                                            nullptr, 0, nullptr, false);
}

int rvvla_csr5_spmv_f32(const rvvla_csr5* A, float alpha, const float* x, float beta, float* y, void* stream) {
  return csr5_spmv_dispatch<float, float, float, float>(A, alpha, x, beta, y, as_stream(stream), nullptr, nullptr,
                                                        0, nullptr, false);
}

int rvvla_csr5_spmv_mixed(const rvvla_csr5* A, int val_type, float alpha, const float* x, float beta, float* y,
                          void* stream) {
  if (val_type == RVVLA_F32)
    return csr5_spmv_dispatch<float, float, CompF32, double>(A, alpha, x, beta, y, as_stream(stream), nullptr,
                                                             nullptr, 0, nullptr, false);
  if (val_type == RVVLA_BF16)
    return csr5_spmv_dispatch<__nv_bfloat16, float, CompF32, double>(A, alpha, x, beta, y, as_stream(stream),
                                                                     nullptr, nullptr, 0, nullptr, false);
  return fail(RVVLA_ERR_INVALID_ARG, "csr5_spmv_mixed: val_type must be RVVLA_F32 or RVVLA_BF16");
}

}  // extern "C"
