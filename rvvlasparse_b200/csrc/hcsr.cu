// hcsr.cu — spMtxHCSR on sm_100a: the GPU builder (bit-exact with the
// reference's crs_to_HCSR) and y = alpha*A*x + beta*y.
//
// Builder: src/scalar/crs_to_hcsr.cpp:30-135.
//   count   — nonzeros per R x C block (integer atomics on run lengths: the
//             counts are order-independent);
//   classify— kind 0 empty / 1 CSR if rows*p < cnt / 2 COO (:61-77, same
//             double-precision comparison);
//   scan    — block_ptr and row_offset exclusive scans, 30-bit and nnz checks
//             (:79-91);
//   scatter — one warp per block-row walks its rows in order, so entries land
//             in each block in source order exactly as the serial loop
//             (:97-119); CSR blocks get per-row counts, COO blocks local rows;
//   prefix  — in-block inclusive scan of CSR row_ptr (:121-126);
//   flags   — kind into bits 31:30 of row_offset (:130-134).
//
// SpMV: src/scalar/spmv_mtx_hcsr.cpp:22-134.  One CTA per block-row keeps the
// block-row's R partial sums in shared memory (the reference keeps them in y);
// the block-row's non-empty blocks are cut into warp work items of 32 rows
// (CSR block; 1 to 32 lanes per row by the block's mean row length) or 256
// nonzeros (the block-row's COO nonzeros as one stream).  The x window of a
// column block (C entries) is read through L1.  Partial sums of different
// blocks are merged with shared-memory atomics, so the summation order inside
// a row can change from run to run (last-bit differences only).
#include <algorithm>
#include <cstring>
#include <string>
#include <type_traits>

#include "crs_merge.cuh"
#include "crs_stream.cuh"
#include "rvvla_internal.cuh"
#include "scan.cuh"

namespace rvvla {
namespace {

constexpr uint32_t kKindMask = 0x3FFFFFFFu;

// ---------------------------------------------------------------- builder
// One thread per row: counts runs of entries falling in the same column block.
__global__ void hcsr_count_kernel(int64_t m, int64_t R, int64_t C, int64_t b_n, const int* __restrict__ Rst,
                                  const int* __restrict__ Col, int64_t* __restrict__ cnt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int64_t base = (i / R) * b_n;
  int64_t run_j = -1, run = 0;
  for (int k = Rst[i]; k < Rst[i + 1]; ++k) {
    const int64_t j = (int64_t)Col[k] / C;
    if (j != run_j) {
      if (run) atomicAdd((unsigned long long*)&cnt[base + run_j], (unsigned long long)run);
      run_j = j;
      run = 0;
    }
    ++run;
  }
  if (run) atomicAdd((unsigned long long*)&cnt[base + run_j], (unsigned long long)run);
}

// kind and row_offset size per block (crs_to_hcsr.cpp:61-77)
__global__ void hcsr_classify_kernel(int64_t nblocks, int64_t m, int64_t R, int64_t b_n, double bs,
                                     const int64_t* __restrict__ cnt, uint8_t* __restrict__ kind,
                                     int64_t* __restrict__ rsz) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  const int64_t br = b / b_n;
  const int64_t r0 = br * R, r1 = min(r0 + R, m);
  const double rows = double(r1 - r0);
  const int64_t c = cnt[b];
  if (c == 0) { kind[b] = 0; rsz[b] = 0; }
  else if (rows * bs < double(c)) { kind[b] = 1; rsz[b] = r1 - r0 + 1; }
  else { kind[b] = 2; rsz[b] = c; }
}

__global__ void hcsr_offsets_kernel(int64_t nb1, const int64_t* __restrict__ bpx, const int64_t* __restrict__ rox,
                                    int* __restrict__ block_ptr, uint32_t* __restrict__ row_offset) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb1) return;
  block_ptr[b] = (int)bpx[b];
  row_offset[b] = (uint32_t)rox[b];
}

// One warp per block-row; rows in order; per row, lanes take up to 32
// entries at a time.  cursor[j] is the next free slot of block j (shared
// memory when the block-row's b_n cursors fit, else global).
template <int VB, bool SMEM>
__global__ void hcsr_scatter_kernel(int64_t m, int64_t R, int64_t C, int64_t b_n, const int* __restrict__ Rst,
                                    const int* __restrict__ Col, const uint8_t* __restrict__ Val,
                                    const int* __restrict__ block_ptr, const uint32_t* __restrict__ row_offset,
                                    const uint8_t* __restrict__ kind, int* __restrict__ gcursor,
                                    uint16_t* __restrict__ col_idx, uint8_t* __restrict__ values,
                                    uint32_t* __restrict__ row_ptr) {
  extern __shared__ int s_cur[];
  const int64_t br = blockIdx.x;
  const unsigned lane = threadIdx.x;
  const int64_t r0 = br * R, r1 = min(r0 + R, m);
  const int64_t blk0 = br * b_n;
  int* cur = SMEM ? s_cur : gcursor + blk0;
  for (int64_t j = lane; j < b_n; j += 32) cur[j] = block_ptr[blk0 + j];
  __syncwarp();
  for (int64_t i = r0; i < r1; ++i) {
    const int64_t li = i - r0;
    const int kb = Rst[i], ke = Rst[i + 1];
    for (int c0 = kb; c0 < ke; c0 += 32) {
      const int k = c0 + (int)lane;
      const bool valid = k < ke;
      const int64_t col = valid ? (int64_t)Col[k] : 0;
      const int64_t j = valid ? col / C : -1;
      const int64_t jprev = __shfl_up_sync(0xffffffffu, j, 1);
      const bool head = valid && (lane == 0 || jprev != j);
      const unsigned heads = __ballot_sync(0xffffffffu, head);
      const unsigned below = heads & ((2u << lane) - 1u);
      const int hl = below ? 31 - __clz(below) : 0;  // lane of my run's head
      // run end: next head or end of the valid lanes
      const unsigned above = heads & ~((2u << lane) - 1u);
      const unsigned vmask = __ballot_sync(0xffffffffu, valid);
      const int nvalid = __popc(vmask);
      const int next_head = above ? __ffs(above) - 1 : nvalid;
      int base = 0;
      if (head) base = cur[j];
      base = __shfl_sync(0xffffffffu, base, hl);
      __syncwarp();
      if (valid) {
        const int64_t blk = blk0 + j;
        const int p = base + ((int)lane - hl);
        col_idx[p] = (uint16_t)(col - j * C);
#pragma unroll
        for (int q = 0; q < VB; ++q) values[(int64_t)p * VB + q] = Val[(int64_t)k * VB + q];
        const uint32_t ro = row_offset[blk];
        if (kind[blk] == 1) {
          if (head) row_ptr[ro + li + 1] += (uint32_t)(next_head - hl);
        } else {
          row_ptr[ro + (p - block_ptr[blk])] = (uint32_t)li;
        }
        if (head) cur[j] = base + (next_head - hl);
      }
      __syncwarp();
    }
  }
}

// In-block inclusive scan of CSR row_ptr (crs_to_hcsr.cpp:121-126); one warp
// per block.
__global__ void hcsr_prefix_kernel(int64_t nblocks, int64_t m, int64_t R, int64_t b_n,
                                   const uint8_t* __restrict__ kind, const uint32_t* __restrict__ row_offset,
                                   uint32_t* __restrict__ row_ptr) {
  const int64_t b = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const unsigned lane = threadIdx.x & 31;
  if (b >= nblocks || kind[b] != 1) return;
  const int64_t br = b / b_n;
  const int64_t rows = min(R, m - br * R);
  uint32_t* rp = row_ptr + row_offset[b];
  uint32_t carry = 0;
  for (int64_t c0 = 1; c0 <= rows; c0 += 32) {
    const int64_t q = c0 + lane;
    uint32_t v = q <= rows ? rp[q] : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t o = __shfl_up_sync(0xffffffffu, v, d);
      if ((int)lane >= d) v += o;
    }
    if (q <= rows) rp[q] = v + carry;
    carry += __shfl_sync(0xffffffffu, v, 31);
  }
}

__global__ void hcsr_flags_kernel(int64_t nblocks, const uint8_t* __restrict__ kind, uint32_t* __restrict__ row_offset) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nblocks) row_offset[b] |= (uint32_t)kind[b] << 30;
}

// ---------------------------------------------------------------- SpMV
template <class Ac> struct HcsrAcc;
template <> struct HcsrAcc<double> { using S = double; };
template <> struct HcsrAcc<float> { using S = float; };

__device__ __forceinline__ float ldx(const float* p) { return __ldg(p); }
__device__ __forceinline__ double ldx(const double* p) { return __ldg(p); }
template <class V> __device__ __forceinline__ V ldv(const V* p) { return __ldg(p); }
template <> __device__ __forceinline__ __nv_bfloat16 ldv<__nv_bfloat16>(const __nv_bfloat16* p) {
  return __ushort_as_bfloat16(__ldg((const unsigned short*)p));
}
__device__ __forceinline__ float to_float(float v) { return v; }
__device__ __forceinline__ float to_float(__nv_bfloat16 v) { return __bfloat162float(v); }

// Finds j with pre[j] <= v < pre[j+1] in a non-decreasing shared array of
// n+1 entries (pre[0] = 0 <= v < pre[n]).
__device__ __forceinline__ int find_slot(const int* pre, int n, int v) {
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pre[mid] <= v) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Number of lanes l whose (non-decreasing across lanes) value b_l is <= q,
// for each lane's own q: a binary search over the warp by shuffles.
__device__ __forceinline__ int warp_count_le(int b, int q) {
  const int b31 = __shfl_sync(0xffffffffu, b, 31);
  int lo = 0;
#pragma unroll
  for (int step = 16; step >= 1; step >>= 1) {
    const int v = __shfl_sync(0xffffffffu, b, lo + step - 1);
    if (v <= q) lo += step;
  }
  if (lo == 31 && b31 <= q) lo = 32;
  return lo;
}

template <class V>
__device__ __forceinline__ V ldval(const V* p, uint64_t pol) { return ld_stream(p, pol); }

template <bool MIX, class V, class X>
__device__ __forceinline__ auto hprod(V v, X x) {
  if constexpr (MIX) return to_float(v) * (float)x;
  else return v * x;
}

// V stored value, X vector type, SA shared accumulator type, MIX: compensated
// fp32 row sums merged into fp64.
//
// Work items of a block-row: every CSR block gives ceil(rows/32) items of 32
// rows (a lane sums one row of the block); all COO nonzeros of the block-row,
// taken block after block, form one stream cut into items of 128 nonzeros (a
// lane finds the block of each of its 4 nonzeros by a shuffle search over the
// COO prefix).  Tiny COO blocks therefore share warps instead of idling them.
// The block-row's prefixes, block starts and row_ptr offsets are staged in
// shared memory first, so an item's loads depend on no other global load; an
// item issues the loads of kHcsrU chunks of 32 nonzeros before using any.
constexpr int kHcsrThreads = 512;
constexpr int kHcsrWarps = kHcsrThreads / 32;
constexpr int kHcsrU = 4;
constexpr int kHcsrSlots = 4;  // loads in flight per lane in a CSR item
// CTAs per SM the register budget is set for.  With 8-byte shared
// accumulators (fp64, and the fp64 merge of the mixed forms) three CTAs (at
// most 40 registers a thread; the few spills stay in L1) hide the gather
// latency better than the registers a two-CTA limit would leave; plain fp32
// sums measured faster at two.
template <class SA>
constexpr int hcsr_min_blocks() { return sizeof(SA) == 8 ? 3 : 2; }

// 32 rows of a CSR block (local rows li0.., nr of them), G = 2^LG lanes per
// row: a group strides through its row's contiguous nonzeros, so one warp
// load covers 32/G rows with G consecutive entries each.  Lane l holds the
// start of row l in rs (e_end: the end of the last row).  The item's rows
// are taken PP passes at a time, each lane issuing kHcsrSlots loads (U per
// row) before using any; longer rows finish in a tail loop.  The group is
// summed by shuffles (fixed butterfly order) and lane gi == 0 adds the row's
// piece to the block-row accumulator in shared memory.
template <int LG, class V, class X, class SA, bool MIX>
__device__ __forceinline__ void hcsr_csr_item(int rs, int e_beg, int e_end, int nr, int li0, int lane, int bp,
                                              const V* __restrict__ values, const uint16_t* __restrict__ col_idx,
                                              const X* __restrict__ xb, SA* acc) {
  using Ac = std::conditional_t<MIX, CompF32, SA>;
  using PT = decltype(hprod<MIX>(V(), X()));
  constexpr int G = 1 << LG, RPP = 32 >> LG, PP = G < 4 ? G : 4, U = kHcsrSlots / PP;
  const int gi = lane & (G - 1);
  for (int p0 = 0; p0 < G; p0 += PP) {
    if (p0 * RPP >= nr) break;
    int st[PP], en[PP];
#pragma unroll
    for (int q = 0; q < PP; ++q) {
      const int r = (p0 + q) * RPP + (lane >> LG);
      const int a = __shfl_sync(0xffffffffu, rs, r & 31);
      const int b = __shfl_sync(0xffffffffu, rs, (r + 1) & 31);
      st[q] = r < nr ? a : 0;
      en[q] = r < nr ? (r + 1 < nr ? b : e_end) : 0;
    }
    PT pv[PP][U];
#pragma unroll
    for (int q = 0; q < PP; ++q)
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = st[q] + gi + u * G;
        const int ei = e < en[q] ? e : e_beg;  // an in-range index for idle slots
        pv[q][u] = hprod<MIX>(ldv(values + bp + ei), ldx(xb + col_idx[bp + ei]));
      }
#pragma unroll
    for (int q = 0; q < PP; ++q) {
      Ac pr;
      acc_zero(pr);
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (st[q] + gi + u * G < en[q]) acc_add(pr, pv[q][u]);
      for (int e = st[q] + gi + U * G; e < en[q]; e += G)
        acc_add(pr, hprod<MIX>(ldv(values + bp + e), ldx(xb + col_idx[bp + e])));
#pragma unroll
      for (int d = 1; d < G; d <<= 1) acc_merge(pr, acc_shfl_xor(pr, d));
      const int r = (p0 + q) * RPP + (lane >> LG);
      if (gi == 0 && r < nr) atomicAdd(&acc[li0 + r], (SA)acc_carry(pr));
    }
  }
}

template <class V, class X, class SA, bool MIX>
__global__ void __launch_bounds__(kHcsrThreads, hcsr_min_blocks<SA>())
hcsr_spmv_kernel(int64_t R, int64_t C, int64_t m, int64_t b_n, const int* __restrict__ block_ptr,
                 const uint32_t* __restrict__ row_offset, const uint32_t* __restrict__ row_ptr,
                 const uint16_t* __restrict__ col_idx, const V* __restrict__ values, const X* __restrict__ x,
                 X* __restrict__ y, X alpha, X beta) {
  using Ac = std::conditional_t<MIX, CompF32, SA>;
  extern __shared__ __align__(16) unsigned char smem[];
  SA* acc = reinterpret_cast<SA*>(smem);
  int* csr_pre = reinterpret_cast<int*>(smem + ((R * sizeof(SA) + 15) / 16) * 16);
  int* coo_pre = csr_pre + (b_n + 1);
  int* s_bp = coo_pre + (b_n + 1);                              // block_ptr of block j (b_n + 1)
  uint32_t* s_off = reinterpret_cast<uint32_t*>(s_bp + b_n + 1);  // row_ptr offset of block j
  __shared__ int s_w[2][kHcsrWarps];
  const int64_t br = blockIdx.x;
  const int64_t r0 = br * R;
  const int maxr = (int)min(R, m - r0);
  const int64_t blk0 = br * b_n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int li = tid; li < maxr; li += kHcsrThreads) acc[li] = SA(0);
  const int row_items = (maxr + 31) >> 5;
  int carry_a = 0, carry_b = 0;
  if (tid == 0) { csr_pre[0] = 0; coo_pre[0] = 0; s_bp[b_n] = block_ptr[blk0 + b_n]; }
  for (int64_t j0 = 0; j0 < b_n; j0 += kHcsrThreads) {
    const int64_t j = j0 + tid;
    int a = 0, b = 0;
    if (j < b_n) {
      const uint32_t ro = row_offset[blk0 + j];
      const int bp = block_ptr[blk0 + j];
      const int nzb = block_ptr[blk0 + j + 1] - bp;
      s_bp[j] = bp;
      s_off[j] = ro & kKindMask;
      if ((ro >> 30) == 1) a = row_items;
      else b = nzb;
    }
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int oa = __shfl_up_sync(0xffffffffu, a, d);
      const int ob = __shfl_up_sync(0xffffffffu, b, d);
      if (lane >= d) { a += oa; b += ob; }
    }
    if (lane == 31) { s_w[0][warp] = a; s_w[1][warp] = b; }
    __syncthreads();
    int wa = 0, wb = 0, ta = 0, tb = 0;
    for (int w = 0; w < kHcsrWarps; ++w) {
      if (w < warp) { wa += s_w[0][w]; wb += s_w[1][w]; }
      ta += s_w[0][w];
      tb += s_w[1][w];
    }
    if (j < b_n) { csr_pre[j + 1] = carry_a + wa + a; coo_pre[j + 1] = carry_b + wb + b; }
    carry_a += ta;
    carry_b += tb;
    __syncthreads();
  }
  const int n_csr = carry_a, n_coo = carry_b;
  const int total = n_csr + (n_coo + 32 * kHcsrU - 1) / (32 * kHcsrU);
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  for (int item = warp; item < total; item += kHcsrWarps) {
    if (item < n_csr) {
      // 32 rows of a CSR block; lanes per row from the block's mean row
      // length (each lane of a group gets about two nonzeros per row)
      const int64_t j = find_slot(csr_pre, (int)b_n, item);
      const int part = item - csr_pre[j];
      const uint32_t off = s_off[j];
      const int bp = s_bp[j];
      const int li0 = part * 32;
      const int nr = min(32, maxr - li0);
      const int mean = (s_bp[j + 1] - bp) / max(maxr, 1);
      const int lg = mean < 4 ? 0 : mean < 8 ? 1 : mean < 16 ? 2 : mean < 32 ? 3 : mean < 64 ? 4 : 5;
      const int rs = (lane < nr) ? (int)row_ptr[off + li0 + lane] : 0;
      const int e_end = (int)row_ptr[off + li0 + nr];
      const int e_beg = __shfl_sync(0xffffffffu, rs, 0);
      if (e_beg < e_end) {
        const X* xb = x + j * C;
        switch (lg) {
#define HCSR_ITEM(L)                                                                                          \
  case L:                                                                                                     \
    hcsr_csr_item<L, V, X, SA, MIX>(rs, e_beg, e_end, nr, li0, lane, bp, values, col_idx, xb, acc);           \
    break;
          HCSR_ITEM(0)
          HCSR_ITEM(1)
          HCSR_ITEM(2)
          HCSR_ITEM(3)
          HCSR_ITEM(4)
          HCSR_ITEM(5)
#undef HCSR_ITEM
        }
      }
    } else {
      // 128 COO nonzeros of the block-row (blocks taken in order): lane 0
      // finds the block of the first one, lanes hold the next 32 block
      // boundaries and a shuffle search places every nonzero.  Nonzeros of
      // a block are in row order, so each chunk of 32 is summed per run of
      // equal rows first and one shared-memory add per run remains.
      const int q0 = (item - n_csr) * (32 * kHcsrU);
      int j0 = 0;
      if (lane == 0) j0 = find_slot(coo_pre, (int)b_n, q0);
      j0 = __shfl_sync(0xffffffffu, j0, 0);
      const int bnd = (j0 + 1 + lane <= b_n) ? coo_pre[j0 + 1 + lane] : INT_MAX;
      int li[kHcsrU];
      SA pv[kHcsrU];
#pragma unroll
      for (int u = 0; u < kHcsrU; ++u) {
        const int q = min(q0 + 32 * u + lane, n_coo - 1);
        const int k = warp_count_le(bnd, q);
        const int64_t j = (k == 32) ? find_slot(coo_pre, (int)b_n, q) : j0 + k;  // > 32 blocks in reach
        const int kk = q - coo_pre[j];
        const int e = s_bp[j] + kk;
        li[u] = (int)row_ptr[s_off[j] + kk];
        const X xv = ld_keep(x + j * C + col_idx[e], pl);
        if constexpr (MIX) pv[u] = (SA)(to_float(ldv(values + e)) * (float)xv);
        else pv[u] = (SA)ldval(values + e, pf) * (SA)xv;
      }
#pragma unroll
      for (int u = 0; u < kHcsrU; ++u) {
        if (q0 + 32 * u >= n_coo) break;
        const bool valid = q0 + 32 * u + lane < n_coo;
        const int rprev = __shfl_up_sync(0xffffffffu, li[u], 1);
        const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || li[u] != rprev);
        const SA sc = acc_seg_scan(valid ? pv[u] : SA(0), heads, lane);
        const int last_valid = min(31, n_coo - 1 - (q0 + 32 * u));
        const bool next_head = lane < 31 && ((heads >> (lane + 1)) & 1u);
        if (valid && ((int)lane == last_valid || next_head)) atomicAdd(&acc[li[u]], sc);
      }
    }
  }
  __syncthreads();
  for (int li = tid; li < maxr; li += kHcsrThreads) {
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
  return RVVLA_OK;
}

template <class V, class X, class SA, bool MIX>
int hcsr_spmv_impl(const rvvla_hcsr* A, X alpha, const X* x, X beta, X* y, cudaStream_t st) {
  int rc = hcsr_validate(A, x, y);
  if (rc) return rc;
  if (A->m == 0) return RVVLA_OK;
  const size_t smem = ((size_t)A->R * sizeof(SA) + 15) / 16 * 16 + (size_t)(4 * A->b_n + 3) * sizeof(int);
  if (smem > 220 * 1024)
    return fail(RVVLA_ERR_UNSUPPORTED, "hcsr: R*sizeof(acc) + 16*b_n exceeds 220 KB of shared memory");
  auto kern = hcsr_spmv_kernel<V, X, SA, MIX>;
  if (smem > 48 * 1024) RVVLA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  prefer_shared(kern);
  kern<<<(unsigned)A->b_m, kHcsrThreads, smem, st>>>(A->R, A->C, A->m, A->b_n, A->block_ptr, A->row_offset, A->row_ptr,
                                            A->col_idx, (const V*)A->values, x, y, alpha, beta);
  RVVLA_LAUNCHED("hcsr_spmv_kernel");
  return RVVLA_OK;
}

}  // namespace

int hcsr_build_impl(const rvvla_crs* src, int vb, int64_t R, int64_t C, double p, rvvla_hcsr_owned* out,
                    cudaStream_t st) {
  if (!src || !out) return fail(RVVLA_ERR_INVALID_ARG, "hcsr_build: null argument");
  std::memset(out, 0, sizeof(*out));
  if (R <= 0 || C <= 0) return fail(RVVLA_ERR_INVALID_ARG, "crs_to_HCSR: R and C must be positive");
  if (C > 65536) return fail(RVVLA_ERR_TOO_LARGE, "crs_to_HCSR: C > 65536 does not fit the uint16 col_idx");
  if (vb != 8 && vb != 4 && vb != 2) return fail(RVVLA_ERR_INVALID_ARG, "hcsr_build: val_bytes must be 8, 4 or 2");
  if (src->m < 0 || src->n < 0 || src->nz < 0) return fail(RVVLA_ERR_INVALID_ARG, "hcsr_build: bad sizes");
  const int64_t m = src->m, n = src->n, nz = src->nz;
  const int64_t b_m = (m + R - 1) / R, b_n = (n + C - 1) / C;
  if (b_n != 0 && b_m > ((int64_t)1 << 40) / b_n) return fail(RVVLA_ERR_TOO_LARGE, "crs_to_HCSR: too many blocks");
  const int64_t nblocks = b_m * b_n;
  rvvla_hcsr& h = out->h;
  h.R = R; h.C = C; h.m = m; h.n = n; h.nz = nz; h.b_m = b_m; h.b_n = b_n;
  RVVLA_CUDA(cudaMalloc(&out->block_ptr, (size_t)(nblocks + 1) * sizeof(int32_t)));
  RVVLA_CUDA(cudaMalloc(&out->row_offset, (size_t)(nblocks + 1) * sizeof(uint32_t)));
  Scratch s_cnt, s_kind, s_x;
  RVVLA_CUDA(s_cnt.alloc((size_t)(2 * nblocks + 2) * sizeof(int64_t), st));
  RVVLA_CUDA(s_kind.alloc((size_t)nblocks + 1, st));
  RVVLA_CUDA(s_x.alloc((size_t)(2 * nblocks + 2) * sizeof(int64_t), st));
  int64_t* cnt = s_cnt.as<int64_t>();
  int64_t* rsz = cnt + nblocks + 1;
  int64_t* bpx = s_x.as<int64_t>();
  int64_t* rox = bpx + nblocks + 1;
  uint8_t* kind = s_kind.as<uint8_t>();
  RVVLA_CUDA(cudaMemsetAsync(cnt, 0, (size_t)(nblocks + 1) * sizeof(int64_t), st));
  if (m > 0) {
    hcsr_count_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(m, R, C, b_n, src->Rst, src->Col, cnt);
    RVVLA_LAUNCHED("hcsr_count_kernel");
  }
  if (nblocks > 0) {
    hcsr_classify_kernel<<<(unsigned)((nblocks + 255) / 256), 256, 0, st>>>(nblocks, m, R, b_n, p, cnt, kind, rsz);
    RVVLA_LAUNCHED("hcsr_classify_kernel");
  }
  int rc = exclusive_scan_i64(cnt, bpx, nblocks, st);
  if (rc) return rc;
  rc = exclusive_scan_i64(rsz, rox, nblocks, st);
  if (rc) return rc;
  int64_t tot[2];
  RVVLA_CUDA(cudaMemcpyAsync(&tot[0], bpx + nblocks, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaMemcpyAsync(&tot[1], rox + nblocks, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaStreamSynchronize(st));
  const int64_t accNz = tot[0], accRows = tot[1];
  if (accRows > ((int64_t)1 << 30) - 1)
    return fail(RVVLA_ERR_TOO_LARGE, "crs_to_HCSR: row_ptr has " + std::to_string(accRows) +
                                         " entries, does not fit the 30-bit row_offset field (use larger C or larger p)");
  if (accNz != nz) return fail(RVVLA_ERR_FORMAT, "crs_to_HCSR: nnz mismatch");
  hcsr_offsets_kernel<<<(unsigned)((nblocks + 1 + 255) / 256), 256, 0, st>>>(nblocks + 1, bpx, rox, out->block_ptr,
                                                                              out->row_offset);
  RVVLA_LAUNCHED("hcsr_offsets_kernel");
  RVVLA_CUDA(cudaMalloc(&out->row_ptr, (size_t)std::max<int64_t>(accRows, 1) * sizeof(uint32_t)));
  RVVLA_CUDA(cudaMalloc(&out->col_idx, (size_t)std::max<int64_t>(nz, 1) * sizeof(uint16_t)));
  RVVLA_CUDA(cudaMalloc(&out->values, (size_t)std::max<int64_t>(nz, 1) * vb));
  RVVLA_CUDA(cudaMemsetAsync(out->row_ptr, 0, (size_t)std::max<int64_t>(accRows, 1) * sizeof(uint32_t), st));
  h.row_ptr_len = accRows;
  if (b_m > 0 && nz > 0) {
    const bool smem = b_n * (int64_t)sizeof(int) <= 200 * 1024;
    Scratch s_cur;
    if (!smem) RVVLA_CUDA(s_cur.alloc((size_t)nblocks * sizeof(int), st));
    const size_t shm = smem ? (size_t)b_n * sizeof(int) : 0;
#define HCSR_SCATTER(VB, SM)                                                                                   \
  do {                                                                                                         \
    auto k_ = hcsr_scatter_kernel<VB, SM>;                                                                     \
    if (shm > 48 * 1024) RVVLA_CUDA(cudaFuncSetAttribute(k_, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm)); \
    k_<<<(unsigned)b_m, 32, shm, st>>>(m, R, C, b_n, src->Rst, src->Col, (const uint8_t*)src->Val,            \
                                        out->block_ptr, out->row_offset, kind, s_cur.as<int>(), out->col_idx,  \
                                        (uint8_t*)out->values, out->row_ptr);                                  \
  } while (0)
    if (vb == 8) { if (smem) HCSR_SCATTER(8, true); else HCSR_SCATTER(8, false); }
    else if (vb == 4) { if (smem) HCSR_SCATTER(4, true); else HCSR_SCATTER(4, false); }
    else { if (smem) HCSR_SCATTER(2, true); else HCSR_SCATTER(2, false); }
#undef HCSR_SCATTER
    RVVLA_LAUNCHED("hcsr_scatter_kernel");
    hcsr_prefix_kernel<<<(unsigned)((nblocks + 7) / 8), 256, 0, st>>>(nblocks, m, R, b_n, kind, out->row_offset,
                                                                        out->row_ptr);
    RVVLA_LAUNCHED("hcsr_prefix_kernel");
  }
  if (nblocks > 0) {
    hcsr_flags_kernel<<<(unsigned)((nblocks + 255) / 256), 256, 0, st>>>(nblocks, kind, out->row_offset);
    RVVLA_LAUNCHED("hcsr_flags_kernel");
  }
  h.block_ptr = out->block_ptr;
  h.row_offset = out->row_offset;
  h.row_ptr = out->row_ptr;
  h.col_idx = out->col_idx;
  h.values = out->values;
  RVVLA_CUDA(cudaStreamSynchronize(st));
  return RVVLA_OK;
}

}  // namespace rvvla

using namespace rvvla;

extern "C" {

int rvvla_hcsr_build(const rvvla_crs* src, int val_bytes, int64_t R, int64_t C, double p, rvvla_hcsr_owned* out,
                     void* stream) {
  int rc = hcsr_build_impl(src, val_bytes, R, C, p, out, as_stream(stream));
  if (rc && out) {
    std::string keep = rvvla_last_error();
    rvvla_hcsr_free(out);
    set_error(keep);
  }
  return rc;
}

void rvvla_hcsr_free(rvvla_hcsr_owned* h) {
  if (!h) return;
  cudaFree(h->block_ptr);
  cudaFree(h->row_offset);
  cudaFree(h->row_ptr);
  cudaFree(h->col_idx);
  cudaFree(h->values);
  std::memset(h, 0, sizeof(*h));
}

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
