// scan.cu — device-wide exclusive prefix sum of int64 counts, used by the GPU
// format builders (block offsets, slice offsets, tile offsets).
// Three passes: per-chunk sums, a single-CTA scan of the chunk sums, then a
// per-chunk block scan seeded with the chunk offset.  out has n+1 entries;
// out[n] is the total.
#include "rvvla_internal.cuh"
#include "scan.cuh"

namespace rvvla {
namespace {

constexpr int kScanThreads = 512;
constexpr int kScanPer = 8;
constexpr int kChunk = kScanThreads * kScanPer;

__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t* s_warp, int64_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t inc = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int64_t o = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += o;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int64_t w = (lane < (int)(blockDim.x >> 5)) ? s_warp[lane] : 0;
    int64_t wi = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      int64_t o = __shfl_up_sync(0xffffffffu, wi, d);
      if (lane >= d) wi += o;
    }
    if (lane < (int)(blockDim.x >> 5)) s_warp[lane] = wi - w;
    if (lane == 31) *total = wi;
  }
  __syncthreads();
  return inc - v + s_warp[warp];
}

__global__ void chunk_sum_kernel(const int64_t* __restrict__ in, int64_t n, int64_t* __restrict__ sums) {
  __shared__ int64_t s_warp[32];
  __shared__ int64_t s_tot;
  const int64_t base = (int64_t)blockIdx.x * kChunk;
  int64_t v = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    int64_t i = base + (int64_t)threadIdx.x * kScanPer + k;
    if (i < n) v += in[i];
  }
  block_excl_scan(v, s_warp, &s_tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = s_tot;
}

__global__ void sums_scan_kernel(int64_t* __restrict__ sums, int64_t nchunks) {
  __shared__ int64_t s_warp[32];
  __shared__ int64_t s_tot;
  int64_t carry = 0;
  for (int64_t b = 0; b < nchunks; b += blockDim.x) {
    int64_t i = b + threadIdx.x;
    int64_t v = i < nchunks ? sums[i] : 0;
    int64_t ex = block_excl_scan(v, s_warp, &s_tot);
    if (i < nchunks) sums[i] = ex + carry;
    carry += s_tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[nchunks] = carry;
}

__global__ void chunk_scan_kernel(const int64_t* __restrict__ in, int64_t n, const int64_t* __restrict__ sums,
                                  int64_t* __restrict__ out) {
  __shared__ int64_t s_warp[32];
  __shared__ int64_t s_tot;
  const int64_t base = (int64_t)blockIdx.x * kChunk + (int64_t)threadIdx.x * kScanPer;
  int64_t loc[kScanPer];
  int64_t v = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    loc[k] = (base + k < n) ? in[base + k] : 0;
    v += loc[k];
  }
  int64_t ex = block_excl_scan(v, s_warp, &s_tot) + sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    if (base + k < n) out[base + k] = ex;
    ex += loc[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = sums[gridDim.x];
}

}  // namespace

int exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t st) {
  if (n <= 0) {
    RVVLA_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), st));
    return RVVLA_OK;
  }
  const int64_t nchunks = (n + kChunk - 1) / kChunk;
  Scratch sc;
  RVVLA_CUDA(sc.alloc((size_t)(nchunks + 1) * sizeof(int64_t), st));
  chunk_sum_kernel<<<(unsigned)nchunks, kScanThreads, 0, st>>>(in, n, sc.as<int64_t>());
  RVVLA_LAUNCHED("chunk_sum_kernel");
  sums_scan_kernel<<<1, 1024, 0, st>>>(sc.as<int64_t>(), nchunks);
  RVVLA_LAUNCHED("sums_scan_kernel");
  chunk_scan_kernel<<<(unsigned)nchunks, kScanThreads, 0, st>>>(in, n, sc.as<int64_t>(), out);
  RVVLA_LAUNCHED("chunk_scan_kernel");
  return RVVLA_OK;
}

}  // namespace rvvla
