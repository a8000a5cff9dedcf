// oracle.h — CPU restatement of RVVLASparse's SpMV path.  TEST INFRASTRUCTURE
// ONLY: tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg are the
// only users.  The product (rvvlasparse_b200) never links or calls this.
//
// Parity status (which parts are pinned by the real reference):
//   * CRS / HCSR / SELL-C-sigma / LAV / CVR SpMV and the CRS->HCSR builder are
//     pinned: tests compare them against the reference scalar library compiled
//     from its own sources (oracle/_ref) and against tests/golden/ fixtures it
//     wrote.
//   * CSR5, VHCC and VNEC (D/S/L) SpMV exist in the reference only as RVV
//     intrinsics (src/rvv/).  Those files compile unmodified against the
//     scalar intrinsic stand-in rvv_emul/riscv_vector.h
//     (oracle/_ref/libref_rvv.so), and tests run them on this oracle's
//     layouts (for VNEC the shim also sets the structures its kernels read,
//     which no reference code fills): all three are pinned.
//   * The reference ships no builder for SELL-C-sigma, CSR5, LAV, VNEC S/D,
//     VHCC or CVR.  The builders here define the layout each reference kernel
//     reads; they are pinned by round trips (format -> CSR == source) and by
//     the reference kernels run on their output (SELL, LAV, CVR, CSR5, VHCC
//     via oracle/_ref).  Parity of those builders is unpinned by the
//     reference.
//
// All formats travel as a "bundle": a format tag, named typed arrays and named
// scalars, so one ctypes binding serves every format.
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

// dtype codes shared with oracle/__init__.py
enum { ORC_I32 = 0, ORC_U32 = 1, ORC_U16 = 2, ORC_U8 = 3, ORC_F32 = 4, ORC_F64 = 5, ORC_I64 = 6, ORC_U64 = 7 };

void* orc_bundle_new(const char* fmt);
void orc_bundle_free(void* h);
const char* orc_bundle_fmt(void* h);
void orc_bundle_put(void* h, const char* name, int dtype, const void* data, int64_t len);
int orc_bundle_count(void* h);
const char* orc_bundle_name(void* h, int i);
int orc_bundle_dtype(void* h, int i);
int64_t orc_bundle_len(void* h, int i);
const void* orc_bundle_data(void* h, int i);
void orc_bundle_set(void* h, const char* name, double v);
int orc_bundle_nscalars(void* h);
const char* orc_bundle_scalar_name(void* h, int i);
double orc_bundle_scalar(void* h, int i);
const char* orc_last_error(void);

// Builders: take a "crs" bundle (Rst i32, Col i32, Val f32|f64; m, n, nz).
// Return a new bundle, or NULL with orc_last_error() set.
void* orc_build_hcsr(void* crs, int64_t R, int64_t C, double p);
void* orc_build_sell(void* crs, int64_t C, int64_t sigma);
void* orc_build_csr5(void* crs, int64_t omega, int64_t sigma);
void* orc_build_lav(void* crs, int64_t simd_lanes, double T, int64_t segment_len);
void* orc_build_vnec(void* crs, int64_t nthreads, int64_t force_variant /* -1 auto, 0 D, 1 S, 2 L */);
void* orc_build_vhcc(void* crs, int64_t nthreads, int64_t vec_size);
void* orc_build_cvr(void* crs, int64_t simd_len, int64_t nthreads);
// Format -> CSR reconstruction (round-trip check), returns a "crs" bundle.
void* orc_to_crs(void* fmt);
// Transposed CSR (counting sort, stable in source order) with the permutation
// perm[k_t] = source position of transposed entry k_t.
void* orc_transpose(void* crs);

// y <- alpha * A b + beta y in the bundle's value type (b, y of that type).
// stage: 0 PREPARATION, 1 MULT, 2 GET_RESULTS, 3 ALL (only SELL distinguishes).
int orc_spmv(void* fmt, double alpha, const void* b, double beta, void* y, int stage);
// Long-double accumulation CSR: y = alpha*A b + beta*y, all in fp64 storage.
void orc_crs_spmv_ld(void* crs, double alpha, const double* b, double beta, double* y);
// dvalues[k] = g[row(k)] * x[col(k)] on the CSR pattern (fp64).
void orc_sddmm(void* crs, const double* g, const double* x, double* dvals);
// Merge-path split point (src/rvv/spmv_mtx_vnec.cpp:42-71).
void orc_merge_path(int64_t diagonal, const int* a, int64_t a_len, int64_t b_len, int64_t* out_xy);

#ifdef __cplusplus
}
#endif
