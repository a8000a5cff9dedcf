// devsort.cuh — stable device radix sort of (key, value) pairs through CUB,
// with its temporary storage from the stream-ordered pool (the GPU builders).
#pragma once
#include <cub/device/device_radix_sort.cuh>

#include "rvvla_internal.cuh"

namespace rvvla {

// Sorts n pairs by the key bits [0, end_bit), stably (equal keys keep their
// input order).
template <class K, class V>
int radix_sort_pairs(const K* kin, K* kout, const V* vin, V* vout, int64_t n, int end_bit, cudaStream_t st) {
  if (n <= 0) return RVVLA_OK;
  if (n > INT32_MAX) return fail(RVVLA_ERR_TOO_LARGE, "radix_sort_pairs: more than 2^31 - 1 items");
  size_t tb = 0;
  RVVLA_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, vin, vout, (int)n, 0, end_bit, st));
  Scratch tmp;
  RVVLA_CUDA(tmp.alloc(tb, st));
  RVVLA_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, kin, kout, vin, vout, (int)n, 0, end_bit, st));
  return RVVLA_OK;
}

// number of bits that hold v (at least 1)
inline int bits_for(uint64_t v) {
  int b = 1;
  while (b < 64 && (v >> b) != 0) ++b;
  return b;
}

inline unsigned grid_for(int64_t n, int threads = 256) {
  return (unsigned)std::max<int64_t>(1, (n + threads - 1) / threads);
}

}  // namespace rvvla
