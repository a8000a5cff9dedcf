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

}  // namespace SparseMatrixLib
