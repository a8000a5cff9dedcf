// hcsr.cu — spMtxHCSR on sm_100a: the GPU builder, bit-exact with the
// reference's crs_to_HCSR (the SpMV is in hcsr_spmv.cu).
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
#include <algorithm>
#include <cstring>
#include <string>
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

}  // extern "C"
