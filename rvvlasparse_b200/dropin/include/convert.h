// convert.h — convertParams and convert<T, MtxDist, simd>(dist, src, params)
// of the RVVLASparse API (include/convert.h:19-31 of the reference).  Every
// destination format is built on the GPU; the built arrays are copied into
// dist's public fields and kept on the device for sparse_mv.  Parameters:
// HCSR "R", "C" (int), "p" (double); SELL "C", "Sigma" (int); CSR5 "omega"
// (int, 32), "sigma" (int); LAV "SIMD_Lanes", "segment_len" (int), "T"
// (double); VHCC "num_threads" (int); CVR "Nthreads" (int).  Errors throw
// like the reference's HCSR builder: std::invalid_argument for bad
// parameters, std::length_error for sizes beyond the index widths,
// std::runtime_error for device failures.
#pragma once
#include <map>
#include <string>

#include "CRS.h"

namespace SparseMatrixLib {

union convertValue {
  int i;
  double d;
};

struct convertParams {
  std::map<std::string, convertValue> param;
};

template <class T, template <class> class MtxDist, bool simd = true>
void convert(MtxDist<T>& dist, const spMtxCRS<T>& src, const convertParams& params) {
  rvvla_convert(dist, src, params);  // found by argument-dependent lookup
}

// Measuring autotuner (an addition; the reference takes every parameter from
// the caller): builds MtxDist from src for each candidate on the GPU, times
// the product (the mixed-precision one when mixed is set: HCSR, SELL, CSR5
// with float values) and returns the convertParams of the fastest, ready for
// convert().  Candidates: HCSR R = C in {512, 1024, 2000, 4000, 8192}, p 2;
// SELL C 32, Sigma {32, 256, 1024, 8192}; CSR5 sigma {8, 16, 24, 32}; LAV
// segment_len {40000, n/4, n}; VHCC num_threads and CVR Nthreads from the
// nonzero count.  Throws like convert on failure.
template <class T, template <class> class MtxDist>
convertParams autotune(const spMtxCRS<T>& src, bool mixed = false, int iters = 5) {
  const MtxDist<T>* tag = nullptr;
  return rvvla_autotune_for(tag, src, mixed, iters);  // found by argument-dependent lookup
}

}  // namespace SparseMatrixLib
