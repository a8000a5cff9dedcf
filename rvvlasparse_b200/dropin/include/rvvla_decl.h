// rvvla_decl.h — declarations of the drop-in library's per-format overloads,
// which the sparse_mv and convert templates reach by argument-dependent
// lookup.  Each format header declares its own.
#pragma once
#include <vector>

#include "types.h"

#define RVVLA_DROPIN_DECLARE_SPMV(CLS)                                                                          \
  sparse_matrix_status rvvla_sparse_mv(sparse_operation_t op, double alpha, const CLS<double>& A,               \
                                       const std::vector<double>& b, double beta, std::vector<double>& y,       \
                                       sparse_matrix_mv_stage stage);                                           \
  sparse_matrix_status rvvla_sparse_mv(sparse_operation_t op, float alpha, const CLS<float>& A,                 \
                                       const std::vector<float>& b, float beta, std::vector<float>& y,          \
                                       sparse_matrix_mv_stage stage);

#define RVVLA_DROPIN_DECLARE_CONVERT(CLS)                                                    \
  void rvvla_convert(CLS<double>& dist, const spMtxCRS<double>& src, const convertParams& p); \
  void rvvla_convert(CLS<float>& dist, const spMtxCRS<float>& src, const convertParams& p);

// the mixed-precision extension (CRS, HCSR, CSR5, SELL-C-sigma): fp32 values,
// b and y; compensated fp32 sums, fp64 carry merges
#define RVVLA_DROPIN_DECLARE_SPMV_MIXED(CLS)                                                               \
  sparse_matrix_status rvvla_sparse_mv_mixed(sparse_operation_t op, float alpha, const CLS<float>& A,     \
                                             const std::vector<float>& b, float beta, std::vector<float>& y);

// the measuring autotuner (an addition): convertParams of the fastest
// candidate for CLS built from src; the pointer argument only selects CLS
#define RVVLA_DROPIN_DECLARE_TUNE(CLS)                                                                          \
  convertParams rvvla_autotune_for(const CLS<double>* tag, const spMtxCRS<double>& src, bool mixed, int iters); \
  convertParams rvvla_autotune_for(const CLS<float>* tag, const spMtxCRS<float>& src, bool mixed, int iters);
