/* rvvla.h — C ABI of the B200 (sm_100a) SpMV library.
 *
 * This is the drop-in boundary for RVVLASparse's SpMV path.  The reference
 * exposes C++ templates only:
 *
 *   sparse_mv<T, Mtx, simd, stage>(op, alpha, A, descr, b, beta, y)
 *       (include/spmv_mtx.h:21-29 of the reference)
 *   convert<T, MtxDist, simd>(dist, src, params)
 *       (include/convert.h:30-31 of the reference)
 *
 * Each entry point below replaces one explicit specialisation of those
 * templates (cited per function).  The C++ drop-in headers under
 * rvvlasparse_b200/dropin/include keep the reference's template signatures and
 * forward to these functions.
 *
 * Conventions
 *   - All array pointers are DEVICE pointers (cudaMalloc'd or equivalent) on
 *     the current CUDA device; `stream` is a cudaStream_t (NULL = legacy
 *     default stream).  Calls are asynchronous with respect to the host unless
 *     stated otherwise.
 *   - Every function returns an rvvla_status; nothing throws or aborts.
 *     rvvla_last_error() returns a message for the calling thread's last
 *     failure.
 *   - y <- alpha * A * x + beta * y.  With beta == 0, y is not read (BLAS
 *     convention; the reference multiplies y by 0, so NaN/Inf already in y
 *     propagate there and not here).
 *   - Descriptor structs mirror the reference classes' public fields (same
 *     names, same meaning), with device pointers.
 *   - Entry points that need temporary device memory obtain it with
 *     cudaMallocAsync/cudaFreeAsync on `stream` (stream-ordered, from the
 *     device's default memory pool).
 */
#ifndef RVVLA_H
#define RVVLA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status */
typedef enum rvvla_status {
  RVVLA_OK = 0,
  RVVLA_ERR_INVALID_ARG = 1,  /* null pointer, negative size, bad parameter   */
  RVVLA_ERR_CUDA = 2,         /* a CUDA runtime call or kernel launch failed    */
  RVVLA_ERR_FORMAT = 3,       /* the format's arrays violate its invariants     */
  RVVLA_ERR_UNSUPPORTED = 4,  /* parameter combination not implemented          */
  RVVLA_ERR_TOO_LARGE = 5,    /* size exceeds an index width or a fixed limit   */
  RVVLA_ERR_TIMEOUT = 6,      /* a bounded device-side wait expired             */
  RVVLA_ERR_NO_DEVICE = 7     /* no CUDA device / not an sm_100 device          */
} rvvla_status;

/* element types (for mixed-precision storage) */
typedef enum rvvla_dtype { RVVLA_F64 = 0, RVVLA_F32 = 1, RVVLA_BF16 = 2 } rvvla_dtype;

/* sparse_matrix_mv_stage of the reference (include/types.h:33-38) */
typedef enum rvvla_stage {
  RVVLA_STAGE_PREPARATION = 0,
  RVVLA_STAGE_MULT = 1,
  RVVLA_STAGE_GET_RESULTS = 2,
  RVVLA_STAGE_ALL = 3
} rvvla_stage;

const char* rvvla_version(void);
const char* rvvla_status_string(int status);
/* Message of the calling thread's last failing call ("" if none). */
const char* rvvla_last_error(void);
/* Fills cc_major/cc_minor/sm_count of the current device; RVVLA_ERR_NO_DEVICE
 * without one. */
int rvvla_device_info(int* cc_major, int* cc_minor, int* sm_count);
/* Number of kernels this library launched in this process (all entry points). */
uint64_t rvvla_kernel_launch_count(void);
/* cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, stream) followed by a
 * stream synchronisation; for callers that manage memory themselves (the
 * builders hand back library-allocated arrays). */
int rvvla_memcpy(void* dst, const void* src, size_t bytes, void* stream);
/* Synchronises `stream`, then reads and clears the device status word that
 * kernels with bounded waits (the bulk-copy pipelines) set when a wait
 * expires.  *code = 0 and RVVLA_OK when no wait expired since the last call;
 * otherwise *code != 0 and RVVLA_ERR_TIMEOUT (results of that call are
 * invalid). */
int rvvla_device_status(int* code, void* stream);

/* ------------------------------------------------------------ CRS (CSR)
 * spMtxCRS<T> (include/CRS.h:10-20 of the reference): m, n, nz, Rst[m+1],
 * Col[nz], Val[nz].  `plan`, `plan_tiles`, `plan_kind` are optional (NULL /
 * 0 / 0): the analysis written by rvvla_crs_analyze.  Without a plan every
 * call computes a merge-path split itself. */
typedef struct rvvla_crs {
  int64_t m, n, nz;
  const int32_t* Rst;
  const int32_t* Col;
  const void* Val;
  const int32_t* plan;
  int64_t plan_tiles;
  int32_t plan_kind; /* 0: merge-path tiles, 1: warp stream (no empty rows) */
} rvvla_crs;

/* Size in int32 entries of the plan buffer for rvvla_crs_analyze (the tile
 * size depends on the value type: RVVLA_F64 or RVVLA_F32; mixed uses F32). */
int64_t rvvla_crs_plan_len(int64_t m, int64_t nz, int dtype);
/* Analyses the row structure once (synchronises `stream`): matrices without
 * empty rows get the warp-stream split (kind 1: first row of each 2048-
 * nonzero warp range), others the merge-path split of (row ends, nonzeros)
 * (kind 0).  Writes plan[], *plan_tiles and *plan_kind for the descriptor. */
int rvvla_crs_analyze(const rvvla_crs* A, int dtype, int32_t* plan, int64_t* plan_tiles,
                      int32_t* plan_kind, void* stream);

/* sparse_mv<double, spMtxCRS, *> — src/scalar/spmv_mtx_crs.cpp:22-46 */
int rvvla_crs_spmv_f64(const rvvla_crs* A, double alpha, const double* x, double beta, double* y,
                       void* stream);
/* sparse_mv<float, spMtxCRS, *> — src/scalar/spmv_mtx_crs.cpp:48-71 */
int rvvla_crs_spmv_f32(const rvvla_crs* A, float alpha, const float* x, float beta, float* y,
                       void* stream);
/* Mixed precision (no reference counterpart): Val stored as val_type
 * (RVVLA_F32 or RVVLA_BF16), x and y fp32, row sums in fp32 with two-sum
 * compensation, cross-tile carries merged in fp64. */
int rvvla_crs_spmv_mixed(const rvvla_crs* A, int val_type, float alpha, const float* x, float beta,
                         float* y, void* stream);

/* ------------------------------------------------------------ HCSR
 * spMtxHCSR<T> (include/HCSR.h:39-53): R, C, m, n, nz, b_m, b_n,
 * block_ptr[b_m*b_n+1] (int), row_offset[b_m*b_n+1] (uint32, kind in bits
 * 31:30: 0 empty, 1 CSR, 2 COO), row_ptr (uint32), col_idx (uint16),
 * values. */
typedef struct rvvla_hcsr {
  int64_t R, C, m, n, nz, b_m, b_n;
  const int32_t* block_ptr;
  const uint32_t* row_offset;
  const uint32_t* row_ptr;
  const uint16_t* col_idx;
  const void* values;
  int64_t row_ptr_len;
} rvvla_hcsr;

/* Output of the GPU builder; the library allocates the arrays (cudaMalloc)
 * and rvvla_hcsr_free releases them. */
typedef struct rvvla_hcsr_owned {
  rvvla_hcsr h;
  int32_t* block_ptr;
  uint32_t* row_offset;
  uint32_t* row_ptr;
  uint16_t* col_idx;
  void* values;
} rvvla_hcsr_owned;

/* convert<T, spMtxHCSR, false> — src/scalar/crs_to_hcsr.cpp:30-169, built on
 * the GPU, bit-exact with the reference (same block kinds, offsets, order).
 * val_bytes: 8 (double), 4 (float) or 2 (bf16 copy of an fp32/fp64 source is
 * not done here; values are copied bit for bit).  R, C > 0; p as in the
 * reference.  Errors mirror the reference's exceptions: INVALID_ARG for
 * R == 0 or C == 0, TOO_LARGE for too many blocks or a row_ptr beyond 30
 * bits.  Synchronises `stream` (sizes are read back to allocate). */
int rvvla_hcsr_build(const rvvla_crs* src, int val_bytes, int64_t R, int64_t C, double p,
                     rvvla_hcsr_owned* out, void* stream);
void rvvla_hcsr_free(rvvla_hcsr_owned* h);

/* sparse_mv<double, spMtxHCSR, *> — src/scalar/spmv_mtx_hcsr.cpp:22-134 */
int rvvla_hcsr_spmv_f64(const rvvla_hcsr* A, double alpha, const double* x, double beta,
                        double* y, void* stream);
/* sparse_mv<float, spMtxHCSR, *> — src/scalar/spmv_mtx_hcsr.cpp:22-134 */
int rvvla_hcsr_spmv_f32(const rvvla_hcsr* A, float alpha, const float* x, float beta, float* y,
                        void* stream);
/* Mixed precision (no reference counterpart): values as val_type (F32/BF16),
 * x, y fp32; per-(row, block) sums in fp32 two-sum, merged across column
 * blocks in fp64. */
int rvvla_hcsr_spmv_mixed(const rvvla_hcsr* A, int val_type, float alpha, const float* x,
                          float beta, float* y, void* stream);

/* ------------------------------------------------------------ CSR5
 * spMtxCSR5<T> (include/CSR5.h:57-88): _m, _n, _nnz, _bit_y_offset,
 * _bit_seg_offset, _tile_desc_len, _tail_tile_start, _p, _omega, _sigma,
 * _num_offsets and the arrays _csr_row_pointer, _csr_column_index,
 * _csr_value (full tiles transposed), _csr5_tile_pointer (p+1),
 * _csr5_tile_descriptor ((p-1)*omega*tile_desc_len),
 * _csr5_tile_empty_offset_pointer (p), _csr5_tile_empty_offset.
 * no_empty_rows (not in the reference class): 1 when every row has a
 * nonzero (set by rvvla_csr5_build); 0 is always safe. */
typedef struct rvvla_csr5 {
  int64_t m, n, nnz;
  int32_t bit_y_offset, bit_seg_offset, tile_desc_len, tail_tile_start;
  int32_t p, omega, sigma, num_offsets;
  const int32_t* csr_row_pointer;
  const uint32_t* csr_column_index;
  const void* csr_value;
  const uint32_t* tile_pointer;
  const uint32_t* tile_descriptor;
  const uint32_t* tile_empty_offset_pointer;
  const uint32_t* tile_empty_offset;
  int32_t no_empty_rows;
} rvvla_csr5;

typedef struct rvvla_csr5_owned {
  rvvla_csr5 h;
  int32_t* csr_row_pointer;
  uint32_t* csr_column_index;
  void* csr_value;
  uint32_t* tile_pointer;
  uint32_t* tile_descriptor;
  uint32_t* tile_empty_offset_pointer;
  uint32_t* tile_empty_offset;
} rvvla_csr5_owned;

/* spMtxCSR5::inputCSR + asCSR5 (declared at include/CSR5.h:61-65, never
 * defined in the reference): builds the layout src/rvv/spmv_mtx_csr5.cpp
 * decodes, on the GPU.  omega <= 32 (the SpMV needs omega == 32), sigma > 0.
 * Synchronises `stream`. */
int rvvla_csr5_build(const rvvla_crs* src, int val_bytes, int omega, int sigma,
                     rvvla_csr5_owned* out, void* stream);
void rvvla_csr5_free(rvvla_csr5_owned* h);
/* sparse_mv<double, spMtxCSR5, true> — src/rvv/spmv_mtx_csr5.cpp:498-541 */
int rvvla_csr5_spmv_f64(const rvvla_csr5* A, double alpha, const double* x, double beta,
                        double* y, void* stream);
/* sparse_mv<float, spMtxCSR5, true> — src/rvv/spmv_mtx_csr5.cpp:543-586 */
int rvvla_csr5_spmv_f32(const rvvla_csr5* A, float alpha, const float* x, float beta, float* y,
                        void* stream);
/* Mixed precision (no reference counterpart): values F32/BF16, x, y fp32,
 * lane sums fp32 two-sum, cross-lane and cross-tile merges fp64. */
int rvvla_csr5_spmv_mixed(const rvvla_csr5* A, int val_type, float alpha, const float* x,
                          float beta, float* y, void* stream);

/* ------------------------------------------------------------ workloads
 * Seeded synthetic matrices on the host (OpenMP), written into caller
 * buffers in two calls: first with NULL arrays to learn nz, then with
 * Rst[m+1], Col[nz], Val[nz] (Val as fp64).  Deterministic for a seed and
 * independent of the thread count. */
/* 5-point Laplacian on a g x g grid (diag 4, off-diagonal -1). */
int64_t rvvla_gen_laplace2d(int64_t g, int32_t* Rst, int32_t* Col, double* Val);
/* 27-point stencil on a g^3 periodic grid, values 1 + 0.1*N(0,1). */
int64_t rvvla_gen_stencil27(int64_t g, uint64_t seed, int32_t* Rst, int32_t* Col, double* Val);
/* Power-law rows: length clamp(round(LogNormal(mu, sigma)),1,cap) with
 * mu = ln(mean) - sigma^2/2; each entry 70% within +-band of the diagonal
 * (clipped to [0,n)), 30% uniform; duplicates redrawn; sorted; U[-1,1]. */
int64_t rvvla_gen_powerlaw(int64_t n, double mean, double sigma, int64_t cap, int64_t band,
                           double band_frac, uint64_t seed, int32_t* Rst, int32_t* Col,
                           double* Val);
/* Rows with geometric(p) lengths (>= 1) or Poisson(mean) lengths
 * (dist 0 / 1), uniform distinct columns, values N(0,1) (val_dist 0) or
 * U[-1,1] (val_dist 1). */
int64_t rvvla_gen_random_rows(int64_t m, int64_t n, int dist, double param, int val_dist,
                              uint64_t seed, int32_t* Rst, int32_t* Col, double* Val);
/* n values U[lo, hi) or N(0,1) (normal != 0). */
void rvvla_gen_vector(int64_t n, uint64_t seed, int normal, double lo, double hi, double* out);

#ifdef __cplusplus
}
#endif
#endif /* RVVLA_H */
