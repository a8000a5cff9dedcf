// rvvla_internal.cuh — shared pieces of the sm_100a kernels and the C ABI:
// status plumbing, stream-ordered scratch, cache-policy loads, warp scans.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <atomic>
#include <string>

#include "rvvla.h"

namespace rvvla {

// ------------------------------------------------------------------ status
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* where);
void count_launch(uint64_t n = 1);

#define RVVLA_CUDA(call)                                      \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return ::rvvla::cuda_fail(e_, #call); \
  } while (0)

// Checks the launch that just happened and counts it.
#define RVVLA_LAUNCHED(name)                                         \
  do {                                                               \
    cudaError_t e_ = cudaGetLastError();                             \
    if (e_ != cudaSuccess) return ::rvvla::cuda_fail(e_, name);      \
    ::rvvla::count_launch();                                         \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int sm_count();
// Per-device status word set by kernels whose bounded waits expired.
int* device_status_word();

// Ask for the largest shared-memory carveout for a kernel whose occupancy is
// bounded by its shared memory (set once per kernel instantiation).
template <class K>
inline void prefer_shared(K kernel) {
  static std::atomic<bool> done{false};
  if (!done.load(std::memory_order_relaxed)) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaGetLastError();
    done.store(true, std::memory_order_relaxed);
  }
}

// Stream-ordered temporary buffer (cudaMallocAsync / cudaFreeAsync).
struct Scratch {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  cudaError_t alloc(size_t bytes, cudaStream_t st) {
    s = st;
    if (bytes == 0) bytes = 16;
    return cudaMallocAsync(&p, bytes, st);
  }
  ~Scratch() {
    if (p) cudaFreeAsync(p, s);
  }
  template <class T>
  T* as() const { return reinterpret_cast<T*>(p); }
};

// ------------------------------------------------------------------ loads
// Streaming operands (values, indices) are read once: evict-first in L2 and
// no L1 allocation.  The gathered vector x is re-read across the whole matrix:
// evict-last keeps it resident in the 126 MB L2.  The asm statements are not
// volatile: they are pure reads of data the kernels never write, so the
// compiler may hoist and batch them to keep many loads in flight.
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

template <class T> __device__ __forceinline__ T ld_stream(const T* p, uint64_t pol);
template <> __device__ __forceinline__ double ld_stream<double>(const double* p, uint64_t pol) {
  double v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
template <> __device__ __forceinline__ float ld_stream<float>(const float* p, uint64_t pol) {
  float v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
template <> __device__ __forceinline__ int ld_stream<int>(const int* p, uint64_t pol) {
  int v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
template <> __device__ __forceinline__ unsigned ld_stream<unsigned>(const unsigned* p, uint64_t pol) {
  unsigned v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
template <> __device__ __forceinline__ unsigned short ld_stream<unsigned short>(const unsigned short* p, uint64_t pol) {
  unsigned short v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b16 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(pol));
  return v;
}
template <> __device__ __forceinline__ __nv_bfloat16 ld_stream<__nv_bfloat16>(const __nv_bfloat16* p, uint64_t pol) {
  unsigned short v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b16 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(pol));
  return __ushort_as_bfloat16(v);
}
__device__ __forceinline__ int4 ld_stream_v4(const int4* p, uint64_t pol) {
  int4 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.b32 {%0,%1,%2,%3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p), "l"(pol));
  return v;
}

template <class T> __device__ __forceinline__ T ld_keep(const T* p, uint64_t pol);
template <> __device__ __forceinline__ double ld_keep<double>(const double* p, uint64_t pol) {
  double v;
  asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
template <> __device__ __forceinline__ float ld_keep<float>(const float* p, uint64_t pol) {
  float v;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}

// value conversion for mixed storage
template <class V> __device__ __forceinline__ float to_f32(V v);
template <> __device__ __forceinline__ float to_f32<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f32<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

// ------------------------------------------------------------------ two-sum
// Compensated fp32 accumulation (Knuth's TwoSum): s + c carries the running
// sum with the rounding error of every addition kept in c.
struct CompF32 {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float v) {
    float t = s + v;
    float bp = t - s;
    float err = (s - (t - bp)) + (v - bp);
    s = t;
    c += err;
  }
  __device__ __forceinline__ void add(const CompF32& o) {
    add(o.s);
    c += o.c;
  }
  __device__ __forceinline__ float value() const { return s + c; }
};

// ------------------------------------------------------------------ warp scan
// Inclusive segmented sum over the warp: lanes with head=true start a new
// segment.  Works for any type with operator+.
template <class T>
__device__ __forceinline__ T warp_seg_scan(T v, bool head, unsigned lane) {
  unsigned heads = __ballot_sync(0xffffffffu, head);
  // distance to the segment's first lane
  unsigned below = heads & ((2u << lane) - 1u);  // heads at lanes <= lane
  int seg_start = below ? (31 - __clz(below)) : 0;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T o = __shfl_up_sync(0xffffffffu, v, d);
    if ((int)lane - d >= seg_start) v = v + o;
  }
  return v;
}

}  // namespace rvvla
