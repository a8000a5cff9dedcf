#pragma once
#include "rvvla_internal.cuh"

namespace rvvla {
// out[0..n] = exclusive prefix sums of in[0..n), out[n] = total.
int exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t st);
}  // namespace rvvla
