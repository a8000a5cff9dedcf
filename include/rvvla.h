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
  RVVLA_ERR_NO_DEVICE = 7,    /* no CUDA device / not an sm_100 device          */
  RVVLA_ERR_IO = 8            /* a file could not be opened, read or written    */
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
/* cudaMalloc / cudaFree on the current device, for host code (the C++
 * drop-in) that keeps device copies without linking the CUDA runtime itself.
 * rvvla_malloc of 0 bytes yields NULL. */
int rvvla_malloc(void** ptr, size_t bytes);
int rvvla_free(void* ptr);
/* Copies from pageable host memory to the device (no reference counterpart:
 * the reference's vectors never leave the host).  Large copies go through
 * the library's page-locked staging buffers in 4 MB chunks, the host memcpy
 * of one chunk (several threads) overlapping the DMA of the previous one.
 * Returns once `src` may be reused; the transfer is ordered on `stream`
 * before later work there. */
int rvvla_copy_h2d(void* dst, const void* src, size_t bytes, void* stream);
/* Device to pageable host memory through the same staging; ordered after
 * earlier work on `stream`, returns once `dst` holds the data. */
int rvvla_copy_d2h(void* dst, const void* src, size_t bytes, void* stream);
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
  int32_t plan_kind; /* 0: merge-path tiles, 1: warp stream, 2: warp stream over non-empty rows */
} rvvla_crs;

/* Size in int32 entries of the plan buffer for rvvla_crs_analyze (the tile
 * size depends on the value type: RVVLA_F64 or RVVLA_F32; mixed uses F32). */
int64_t rvvla_crs_plan_len(int64_t m, int64_t nz, int dtype);
/* Analyses the row structure once (synchronises `stream`) for the lane-run
 * kernel (256 to 2048 nonzeros per warp by matrix size, 8 per lane, plus a
 * row-start bitmap of one bit per nonzero): matrices without empty rows get
 * kind 1 (first row of each warp range; plan_tiles = warps), matrices with
 * empty rows kind 2 (the non-empty rows compacted with a map back to their
 * ids and the list of empty rows; plan_tiles = non-empty rows), matrices
 * without nonzeros the merge-path split of (row ends, nonzeros) (kind 0).
 * Writes plan[], *plan_tiles and *plan_kind for the descriptor. */
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

/* ------------------------------------------------------------ SELL-C-sigma
 * spMtxSELL_C_Sigma<T> (include/SELL_C_Sigma.h:23-40): m, n, cnt_b, nz, C,
 * Sigma, vCl/vCs/vBs/vSBs[cnt_b], vCol/vVal[len], vPerm[m]. */
typedef struct rvvla_sell {
  int64_t m, n, cnt_b, nz;
  int32_t C, Sigma;
  const int32_t* vCl;
  const int32_t* vCs;
  const int32_t* vBs;
  const int32_t* vSBs;
  const uint32_t* vCol;
  const uint32_t* vPerm;
  const void* vVal;
  int64_t len;
} rvvla_sell;

typedef struct rvvla_sell_owned {
  rvvla_sell h;
  int32_t *vCl, *vCs, *vBs, *vSBs;
  uint32_t *vCol, *vPerm;
  void* vVal;
} rvvla_sell_owned;

/* Builder (the reference has none): rows sorted by length, descending and
 * stable, inside windows of sigma rows; slices of C rows; column-major slice
 * storage padded with value 0 / column 0.  Synchronises `stream`. */
int rvvla_sell_build(const rvvla_crs* src, int val_bytes, int64_t C, int64_t sigma,
                     rvvla_sell_owned* out, void* stream);
void rvvla_sell_free(rvvla_sell_owned* h);
/* sparse_mv<double, spMtxSELL_C_Sigma, *, stage> —
 * src/scalar/spmv_mtx_sell_c_sigma.cpp:22-149; stage is an rvvla_stage. */
int rvvla_sell_spmv_f64(const rvvla_sell* A, int stage, double alpha, const double* x, double beta,
                        double* y, void* stream);
/* sparse_mv<float, spMtxSELL_C_Sigma, *, stage> —
 * src/scalar/spmv_mtx_sell_c_sigma.cpp:151-275 */
int rvvla_sell_spmv_f32(const rvvla_sell* A, int stage, float alpha, const float* x, float beta,
                        float* y, void* stream);
/* Mixed precision, all stages (no reference counterpart). */
int rvvla_sell_spmv_mixed(const rvvla_sell* A, int val_type, float alpha, const float* x,
                          float beta, float* y, void* stream);

/* ------------------------------------------------------------ LAV
 * spMtxLAV<T> (include/LAV.h:11-31): SIMD_Lanes, m, n, nz, segment_count,
 * chunk_count, T, segment_len, chunk_offsets[(chunk_count+1)*segment_count],
 * chunk_offsets_full_mask[chunk_count*segment_count],
 * segment_ptr[segment_count+1], out_order[segment_count*chunk_count*SIMD_Lanes],
 * mask[n_steps], val/col_id[n_steps*SIMD_Lanes] and sparse_part (CRS). */
typedef struct rvvla_lav {
  int64_t SIMD_Lanes, m, n, nz, segment_count, chunk_count, segment_len, n_steps;
  double T;
  const int32_t* chunk_offsets;
  const int32_t* chunk_offsets_full_mask;
  const uint64_t* segment_ptr;
  const uint32_t* out_order;
  const uint16_t* mask;
  const void* val;
  const uint32_t* col_id;
  rvvla_crs sparse_part;
  /* Optional (not in the reference class; NULL = one launch per segment):
   * row_order[m] = the global row order the chunks are cut from, and
   * lane_of_slot[(segment*chunk_count + chunk)*SIMD_Lanes + j] = the lane
   * holding row_order[chunk*SIMD_Lanes + j] in that segment.  With them (and
   * SIMD_Lanes dividing 32) one launch walks all segments and updates each
   * row of y once.  long_chunks (0 = none): the leading chunks that get a
   * thread block each, their steps spread over the block (the builder sets
   * it to cover the chunks of >= 128 steps). */
  const uint32_t* row_order;
  const uint8_t* lane_of_slot;
  int64_t long_chunks;
} rvvla_lav;

typedef struct rvvla_lav_owned {
  rvvla_lav h;
  int32_t *chunk_offsets, *chunk_offsets_full_mask;
  uint64_t* segment_ptr;
  uint32_t* out_order;
  uint16_t* mask;
  void* val;
  uint32_t* col_id;
  int32_t *sp_Rst, *sp_Col;
  void* sp_Val;
  uint32_t* row_order;
  uint8_t* lane_of_slot;
  int32_t* sp_plan; /* rvvla_crs_analyze plan of sparse_part (the builder sets h.sparse_part.plan) */
} rvvla_lav_owned;

/* Builder (the reference has none; built on the GPU with stable radix sorts,
 * only the few scalars of the plan pass through the host): dense
 * columns = the most populated columns holding >= (1-T) of the nonzeros,
 * segments of segment_len of them; rows chunked by dense count, descending;
 * inside a chunk each segment orders rows by their count in that segment.
 * Synchronises `stream`. */
int rvvla_lav_build(const rvvla_crs* src, int val_bytes, int64_t simd_lanes, double T,
                    int64_t segment_len, rvvla_lav_owned* out, void* stream);
void rvvla_lav_free(rvvla_lav_owned* h);
/* sparse_mv<double, spMtxLAV, false> — src/scalar/spmv_mtx_lav.cpp:24-85 */
int rvvla_lav_spmv_f64(const rvvla_lav* A, double alpha, const double* x, double beta, double* y,
                       void* stream);
/* sparse_mv<float, spMtxLAV, false> — src/scalar/spmv_mtx_lav.cpp:87-148 */
int rvvla_lav_spmv_f32(const rvvla_lav* A, float alpha, const float* x, float beta, float* y,
                       void* stream);

/* ------------------------------------------------------------ VNEC
 * spMtxVNEC<T> (include/VNEC.h:35-76): the source CRS (ptr/indices/val =
 * M.ptr/M.indices/M.val), NUM_THREADS_VNEC, vnec_t (SpB_VNEC_type: 0 D,
 * 1 S, 2 L), IRD_mat, thread_coord_start/_end ((x, y) pairs per thread),
 * D arrays (ecr_indices, NEC_NUM, use_x_indices (flattened, offsets
 * use_x_ptr), v_row_ptr, col_start, val_align) and S arrays (tasks
 * (flattened), reorder_mat.task_start/task_end/row_begin/row_end/col/nnz,
 * spvv_len).  nLanes = nLanes_f64 (8) or nLanes_f32 (16); max_nec = largest
 * NEC_NUM (the shared-memory size of the compacted x). */
typedef struct rvvla_vnec {
  int64_t m, n, nz;
  int32_t NUM_THREADS_VNEC, nLanes, vnec_t, max_nec;
  float IRD_mat;
  const int32_t* ptr;
  const int32_t* indices;
  const void* val;
  const int32_t* thread_coord_start;
  const int32_t* thread_coord_end;
  const int32_t* ecr_indices;
  const int32_t* NEC_NUM;
  const int32_t* use_x_ptr;
  const int32_t* use_x_indices;
  const int32_t* v_row_ptr;
  const int32_t* col_start;
  const void* val_align;
  int64_t ngroups;
  const int32_t* tasks;
  const int32_t* task_start;
  const int32_t* task_end;
  const int32_t* spvv_len;
  const int32_t* row_begin;
  const int32_t* row_end;
  const int32_t* reorder_col;
  const void* reorder_nnz;
  int64_t ntasks, nreorder;
  /* Optional (not in the reference class): the rvvla_crs_analyze plan of the
   * source CRS for the L variant (NULL = merge path over the VNEC threads'
   * coordinates). */
  const int32_t* plan;
  int64_t plan_tiles;
  int32_t plan_kind;
} rvvla_vnec;

typedef struct rvvla_vnec_owned {
  rvvla_vnec h;
  int32_t *ptr, *indices;
  void* val;
  int32_t *thread_coord_start, *thread_coord_end, *ecr_indices, *NEC_NUM, *use_x_ptr, *use_x_indices;
  int32_t *v_row_ptr, *col_start;
  void* val_align;
  int32_t *tasks, *task_start, *task_end, *spvv_len, *row_begin, *row_end, *reorder_col;
  void* reorder_nnz;
  int32_t* plan;
} rvvla_vnec_owned;

/* spMtxVNEC(const spMtxCRS&) (include/VNEC.h:200-227): partition, x
 * compaction, IRD and variant choice, plus the S/D structures the
 * reference's kernels read (built on the GPU: merge-path partition, compaction
 * by a stable radix sort, per-group and per-task scans; the IRD and the
 * variant choice read a few scalars back).  nthreads <= 0
 * picks one merge tile (2048 items) per thread; variant -1 applies the
 * reference's rule, 0/1/2 force D/S/L.  val_bytes 8 or 4.  Synchronises
 * `stream`. */
int rvvla_vnec_build(const rvvla_crs* src, int val_bytes, int64_t nthreads, int variant,
                     rvvla_vnec_owned* out, void* stream);
void rvvla_vnec_free(rvvla_vnec_owned* h);
/* sparse_mv<double, spMtxVNEC, true> — src/rvv/spmv_mtx_vnec.cpp:588-657 */
int rvvla_vnec_spmv_f64(const rvvla_vnec* A, double alpha, const double* x, double beta,
                        double* y, void* stream);
/* sparse_mv<float, spMtxVNEC, true> — src/rvv/spmv_mtx_vnec.cpp:659-738 */
int rvvla_vnec_spmv_f32(const rvvla_vnec* A, float alpha, const float* x, float beta, float* y,
                        void* stream);

/* ------------------------------------------------------------ VHCC
 * spMtxVHCC<T> (include/VHCC.h:15-60): vhcc_params (num_threads,
 * num_panels, tile_row, tile_col, vec_size, n_masks), _num_rows, _num_cols,
 * _num_entries, _num_vectors, _pad_entries, _pad_rows, _thr_info
 * (num_threads x 10 ints: vbase, rbase, sbase, last_row, overflow_row,
 * start_vec, end_vec, panel_id, merge_start, merge_end), _veceor_ptr
 * (n_eor entries incl. the sentinel), _scan_mask (bytes), _row_arr,
 * _col_arr, _vals_arr (num_vectors*vec_size). */
typedef struct rvvla_vhcc {
  int64_t num_rows, num_cols, num_entries, num_vectors, pad_entries, pad_rows;
  int32_t num_threads, num_panels, tile_row, tile_col, vec_size, n_masks;
  const int32_t* thr_info;
  const uint32_t* veceor_ptr;
  int64_t n_eor;
  const uint8_t* scan_mask;
  int64_t scan_mask_bytes;
  const uint32_t* row_arr;
  int64_t n_rowarr;
  const uint32_t* col_arr;
  const void* vals_arr;
} rvvla_vhcc;

typedef struct rvvla_vhcc_owned {
  rvvla_vhcc h;
  int32_t* thr_info;
  uint32_t* veceor_ptr;
  uint8_t* scan_mask;
  uint32_t *row_arr, *col_arr;
  void* vals_arr;
} rvvla_vhcc_owned;

/* Builder (the reference has only setters, include/VHCC.h:80-112): one
 * panel, vec_size 32 (one vector lane per warp lane), num_threads equal
 * vector ranges (<= 0: 64 vectors each).  Synchronises `stream`.
 * Several panels (vhcc_params.num_panels, include/VHCC.h:15-26): build one
 * structure per column range of the CRS (global column indices kept) and
 * call rvvla_vhcc_spmv_* on them in column order, beta on the first and 1
 * after; the Python mirror does this for convertParams(num_panels=P). */
int rvvla_vhcc_build(const rvvla_crs* src, int val_bytes, int64_t num_threads, rvvla_vhcc_owned* out,
                     void* stream);
void rvvla_vhcc_free(rvvla_vhcc_owned* h);
/* sparse_mv<double, spMtxVHCC, true> — src/rvv/spmv_vhcc.cpp:320-434 */
int rvvla_vhcc_spmv_f64(const rvvla_vhcc* A, double alpha, const double* x, double beta,
                        double* y, void* stream);
/* sparse_mv<float, spMtxVHCC, true> — src/rvv/spmv_vhcc.cpp:252-316 */
int rvvla_vhcc_spmv_f32(const rvvla_vhcc* A, float alpha, const float* x, float beta, float* y,
                        void* stream);

/* ------------------------------------------------------------ CVR
 * spMtxCVR<T> (include/CVR.h:22-37): nItems, numRows, numCols, SIMD_LEN,
 * Nthreads, Nthreads_avail, vPack_vec_vals/cols (nItems),
 * vPack_vec_record (n_record ints: (pos, row) pairs + one trailing pair),
 * writeback_pos_record (n_writeback = Nthreads_avail*(SIMD_LEN+2) ints). */
typedef struct rvvla_cvr {
  int64_t nItems, numRows, numCols;
  int32_t SIMD_LEN, Nthreads, Nthreads_avail, no_empty_rows;
  const void* vPack_vec_vals;
  const uint32_t* vPack_vec_cols;
  const int32_t* vPack_vec_record;
  int64_t n_record;
  const int32_t* writeback_pos_record;
  int64_t n_writeback;
} rvvla_cvr;

typedef struct rvvla_cvr_owned {
  rvvla_cvr h;
  void* vPack_vec_vals;
  uint32_t* vPack_vec_cols;
  int32_t *vPack_vec_record, *writeback_pos_record;
} rvvla_cvr_owned;

/* Builder (the reference has none): SIMD_LEN 32; nthreads whole-row
 * ranges balanced by nonzeros (<= 0: 16384 nonzeros each); rows enter lanes
 * longest first.  Synchronises `stream`. */
int rvvla_cvr_build(const rvvla_crs* src, int val_bytes, int64_t nthreads, rvvla_cvr_owned* out,
                    void* stream);
void rvvla_cvr_free(rvvla_cvr_owned* h);
/* sparse_mv<double, spMtxCVR, false> — src/scalar/spmv_mtx_cvr.cpp:21-68 */
int rvvla_cvr_spmv_f64(const rvvla_cvr* A, double alpha, const double* x, double beta, double* y,
                       void* stream);
/* sparse_mv<float, spMtxCVR, false> — src/scalar/spmv_mtx_cvr.cpp:70-118 */
int rvvla_cvr_spmv_f32(const rvvla_cvr* A, float alpha, const float* x, float beta, float* y,
                       void* stream);

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
/* rvvla_csr5_spmv_f64 without any device allocation (no counterpart in the
 * reference): the per-warp calibrator lives in a static device array of
 * 8192 slots (96 KB), enough for every launch on a B200; a matrix whose
 * launch needs more returns RVVLA_ERR_TOO_LARGE.  The first call on each
 * device resolves that array's address (and may load the module): make it
 * before any stream capture.  Calls overlapping in time on one device share
 * the array and race: serialise them.  Always runs the register-staged
 * kernel, whatever RVVLA_CSR5_STAGING selects for the ordinary entry. */
int rvvla_csr5_spmv_f64_noalloc(const rvvla_csr5* A, double alpha, const double* x, double beta,
                                double* y, void* stream);

/* ------------------------------------------------------------ adjoint
 * No reference counterpart (the reference declares SPARSE_OPERATION_TRANSPOSE
 * in include/types.h:24-27 and ignores it).  For y = alpha*A(v)*x with a fixed
 * pattern: dx = A^T g through a transposed CRS built on the GPU, and
 * dv[k] = g[row(k)] * x[Col[k]] on A's pattern (SDDMM). */
typedef struct rvvla_transpose {
  rvvla_crs AT;         /* A^T: n x m CRS, with its analysis plan */
  const int32_t* perm;  /* perm[k] = index in A of A^T's k-th nonzero */
  int32_t val_bytes;    /* element size of AT.Val: 8, 4 or 2 */
} rvvla_transpose;

typedef struct rvvla_transpose_owned {
  rvvla_transpose h;
  int32_t *Rst, *Col, *perm, *plan;
  void* Val;
} rvvla_transpose_owned;

/* Builds A^T (entries of a column in ascending row order) and the
 * permutation; copies A's values when A->Val is not NULL.  Synchronises
 * `stream`. */
int rvvla_csr_transpose(const rvvla_crs* A, int val_bytes, rvvla_transpose_owned* out,
                        void* stream);
void rvvla_csr_transpose_free(rvvla_transpose_owned* h);
/* ValT[k] = Val[perm[k]]: refreshes A^T's values after A's values changed. */
int rvvla_csr_transpose_values(const rvvla_transpose* T, const void* Val, void* ValT,
                               void* stream);
/* dx = alpha * A^T g + beta * dx (the CRS kernels on A^T; beta = 0 does not
 * read dx). */
int rvvla_spmv_adjoint_x_f64(const rvvla_transpose* T, double alpha, const double* g,
                             double beta, double* dx, void* stream);
int rvvla_spmv_adjoint_x_f32(const rvvla_transpose* T, float alpha, const float* g,
                             float beta, float* dx, void* stream);
/* The same product with A's current values Val (nz entries, A's order) read
 * through the transpose's permutation inside the kernel: no
 * rvvla_csr_transpose_values pass, A^T's own value array is not used. */
int rvvla_spmv_adjoint_x_values_f64(const rvvla_transpose* T, const double* Val, double alpha,
                                    const double* g, double beta, double* dx, void* stream);
int rvvla_spmv_adjoint_x_values_f32(const rvvla_transpose* T, const float* Val, float alpha,
                                    const float* g, float beta, float* dx, void* stream);
/* dvalues[k] = g[row(k)] * x[Col[k]] for every nonzero k of A. */
int rvvla_sddmm_values_f64(const rvvla_crs* A, const double* g, const double* x, double* dvalues,
                           void* stream);
int rvvla_sddmm_values_f32(const rvvla_crs* A, const float* g, const float* x, float* dvalues,
                           void* stream);

/* ------------------------------------------------------------ batched
 * No reference counterpart.  Many independent matrices, each with k right-
 * hand sides, in one persistent launch: Y_i = alpha * A_i X_i + beta * Y_i.
 * X_i is n_i x k and Y_i is m_i x k, row-major, packed matrix after matrix
 * (matrix i starts at x_off[i] / y_off[i] elements). */
typedef struct rvvla_batch {
  int64_t count, k, x_len, y_len, ntiles;
  int32_t val_bytes, grid, block;
  const void* mats;   /* device table, one entry per matrix */
  const void* tiles;  /* device work list */
} rvvla_batch;

typedef struct rvvla_batch_owned {
  rvvla_batch h;
  void* mats;
  void* tiles;
  int64_t* x_off;          /* host, count + 1 entries */
  int64_t* y_off;          /* host, count + 1 entries */
  rvvla_sell_owned* sell;  /* host, the SELL copies of mode-1 matrices */
  int64_t nmats;
} rvvla_batch_owned;

/* Plans a batch of CRS matrices (device arrays, which must stay alive):
 * val_bytes 4 or 8; k in {1, 4, 8, 32}; mode[i] 0 = CSR (param[i] = threads
 * per row for k = 1, a power of two <= 32, 0 = by average row length) or
 * 1 = SELL-C-sigma with C = 32 built on the GPU (param[i] = sigma, 0 = 256);
 * mode/param may be NULL (all CSR, default threads per row).  Synchronises
 * `stream`. */
int rvvla_batched_plan(const rvvla_crs* mats, int64_t count, int val_bytes, int k, const int32_t* mode,
                       const int32_t* param, rvvla_batch_owned* out, void* stream);
void rvvla_batched_free(rvvla_batch_owned* b);
/* One persistent launch over all matrices. */
int rvvla_batched_spmv_f64(const rvvla_batch* B, double alpha, const double* X, double beta, double* Y,
                           void* stream);
int rvvla_batched_spmv_f32(const rvvla_batch* B, float alpha, const float* X, float beta, float* Y,
                           void* stream);
/* Captures that launch (fixed alpha, X, beta, Y) into a CUDA graph on a
 * non-default `stream` and instantiates it; *graph is an opaque handle. */
int rvvla_batched_graph(const rvvla_batch* B, double alpha, const void* X, double beta, void* Y,
                        void* stream, void** graph);
int rvvla_batched_graph_launch(void* graph, void* stream);
void rvvla_batched_graph_free(void* graph);
/* ------------------------------------------------------------ autotuner
 * Parameters for convert (the reference's convertParams bag,
 * include/convert.h:21-28, whose keys the drop-in fills from these fields):
 * HCSR "R", "C", "p"; SELL "C", "Sigma"; CSR5 "sigma" (omega 32); LAV
 * "SIMD_Lanes", "T", "segment_len"; VHCC "num_threads"; CVR "Nthreads". */
typedef enum rvvla_format {
  RVVLA_FMT_HCSR = 1,
  RVVLA_FMT_SELL = 2,
  RVVLA_FMT_CSR5 = 3,
  RVVLA_FMT_LAV = 4,
  RVVLA_FMT_VHCC = 5,
  RVVLA_FMT_CVR = 6
} rvvla_format;

typedef struct rvvla_tune_params {
  int64_t R, C;                     /* HCSR block rows/columns; SELL slice height in C */
  double p;                         /* HCSR CSR/COO threshold */
  int64_t sigma;                    /* SELL-C-sigma window; CSR5 sigma */
  int64_t threads;                  /* VHCC num_threads; CVR Nthreads */
  int64_t simd_lanes, segment_len;  /* LAV */
  double T;                         /* LAV dense threshold */
} rvvla_tune_params;

/* Measuring autotuner for one format (no reference counterpart; the
 * reference takes its parameters from the caller).  Builds the format on the
 * GPU from src (values of val_type: RVVLA_F64 / RVVLA_F32, or RVVLA_BF16 with
 * mixed) for each candidate, times the product (plain, or the mixed form
 * when mixed != 0: HCSR, SELL, CSR5) with CUDA events, best of iters after
 * one untimed call, and writes the fastest candidate to *best (and its ms to
 * *best_ms).  table/table_ms (table_cap entries, may be NULL) receive every
 * candidate and its time; *n_candidates the count.  Candidates: HCSR R = C in
 * {512, 1024, 2000, 4000, 8192}, p 2; SELL C 32, sigma {32, 256, 1024, 8192};
 * CSR5 sigma {8, 16, 24, 32}; LAV segment_len {40000, n/4, n}; VHCC
 * nnz / {4096, 2048, 1024} threads; CVR nnz / {8192, 32768, 131072} ranges.
 * Synchronises `stream`. */
int rvvla_autotune(int format, const rvvla_crs* src, int val_type, int mixed, int iters,
                   rvvla_tune_params* best, double* best_ms, rvvla_tune_params* table, double* table_ms,
                   int table_cap, int* n_candidates, void* stream);

/* Autotuner: groups the matrices by average row length (powers of two),
 * times every candidate configuration on each group with CUDA events (CSR
 * with 1..32 threads per row for k = 1 or k lanes per row otherwise;
 * SELL-C-sigma with sigma 32 or 256) and writes the fastest per matrix into
 * mode[] / param[] (count entries each), ready for rvvla_batched_plan.
 * *tuned_ms (may be NULL) receives the sum of the groups' best times. */
int rvvla_batched_autotune(const rvvla_crs* mats, int64_t count, int val_bytes, int k, int32_t* mode,
                           int32_t* param, double* tuned_ms, void* stream);

/* ------------------------------------------------------------ solvers
 * Conjugate gradients for symmetric positive definite A (no reference
 * counterpart: a caller of the SpMV path).  A is square, has nonzeros and an
 * rvvla_crs_analyze plan.  x holds the initial guess and receives the
 * solution; b, x are device vectors.  Each iteration runs q = A p with p.q
 * fused into the SpMV, then x/r updates with the new r.r fused into the
 * same pass; no host synchronisation except a read of r.r every
 * check_every iterations (so up to check_every - 1 iterations may run after
 * convergence).  Stops when ||r|| <= rtol ||b|| (recurrence residual) or
 * after max_iter iterations; *iters and *rel_res = ||r|| / ||b|| report
 * where it stopped (RVVLA_OK either way).  Scratch: 3 vectors of n plus
 * partials, stream-ordered.  Bitwise reproducible. */
int rvvla_cg_f64(const rvvla_crs* A, const double* b, double* x, int64_t max_iter, double rtol,
                 int64_t check_every, int64_t* iters, double* rel_res, void* stream);
int rvvla_cg_f32(const rvvla_crs* A, const float* b, float* x, int64_t max_iter, double rtol,
                 int64_t check_every, int64_t* iters, double* rel_res, void* stream);
/* BiCGStab (van der Vorst) for a general square A, unpreconditioned (no
 * reference counterpart: a caller of the SpMV path).  Same A, x, b, limits
 * and check schedule as rvvla_cg_*; per iteration two CRS products
 * (v = A p, t = A s), the dots r^.v, t.s, t.t, r^.r and r.r reduced in a
 * fixed order, and three fused vector passes, scalars on the device.
 * *breakdown = 1 when it stopped unconverged because r^.r, r^.v or t.t
 * became exactly zero (RVVLA_OK either way).  Scratch: 6 vectors of n plus
 * partials, stream-ordered.  Bitwise reproducible. */
int rvvla_bicgstab_f64(const rvvla_crs* A, const double* b, double* x, int64_t max_iter, double rtol,
                       int64_t check_every, int64_t* iters, double* rel_res, int* breakdown, void* stream);
int rvvla_bicgstab_f32(const rvvla_crs* A, const float* b, float* x, int64_t max_iter, double rtol,
                       int64_t check_every, int64_t* iters, double* rel_res, int* breakdown, void* stream);
/* y = A x and *dot = x^T A x (a device scalar) in one pass over A: the
 * building block of the solver for other Krylov methods.  A square with an
 * rvvla_crs_analyze plan (or without nonzeros: y = 0, *dot = 0); the dot
 * is summed in a fixed order (bitwise reproducible); stream-ordered scratch
 * of one value per 256-2048 nonzeros. */
int rvvla_crs_spmv_dot_f64(const rvvla_crs* A, const double* x, double* y, double* dot, void* stream);
int rvvla_crs_spmv_dot_f32(const rvvla_crs* A, const float* x, float* y, float* dot, void* stream);

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

/* ------------------------------------------------------------ files
 * Host-side sparse matrices on disk (no device involved).  The reference's
 * spMtxCRS carries a Matrix Market type code (include/CRS.h:8,17) but ships
 * no reader, and its test environment names an "mtx to bin" converter
 * (cmake/TestEnvironment.cmake:62); these provide both. */
/* A CRS matrix in host memory allocated by the library (malloc);
 * rvvla_host_crs_free releases the arrays. */
typedef struct rvvla_host_crs {
  int64_t m, n, nz;
  int32_t* Rst;
  int32_t* Col;
  double* Val;
} rvvla_host_crs;
void rvvla_host_crs_free(rvvla_host_crs* A);
/* Reads a Matrix Market coordinate file (real / integer / pattern;
 * general / symmetric / skew-symmetric) into CRS with ascending columns in
 * every row; duplicate entries are summed in file order.  Errors: RVVLA_ERR_IO
 * (unreadable), RVVLA_ERR_FORMAT (malformed, index outside the matrix),
 * RVVLA_ERR_UNSUPPORTED (complex, Hermitian or dense "array" files). */
int rvvla_mm_read(const char* path, rvvla_host_crs* out);
/* Writes a CRS matrix as "matrix coordinate real general" (17 digits). */
int rvvla_mm_write(const char* path, int64_t m, int64_t n, const int32_t* Rst, const int32_t* Col,
                   const double* Val);
/* Binary CRS container: 48-byte header ("RVVLACRS", version 1, value bytes,
 * m, n, nz), then Rst, Col, Val as stored in memory (little-endian). */
int rvvla_crs_save(const char* path, int64_t m, int64_t n, int64_t nz, const int32_t* Rst,
                   const int32_t* Col, const void* Val, int val_bytes);
/* Header of a binary CRS file (checked against the file length). */
int rvvla_crs_load_info(const char* path, int64_t* m, int64_t* n, int64_t* nz, int* val_bytes);
/* Arrays of a binary CRS file into caller buffers sized from
 * rvvla_crs_load_info; the row pointers and columns are validated. */
int rvvla_crs_load(const char* path, int32_t* Rst, int32_t* Col, void* Val);

#ifdef __cplusplus
}
#endif
#endif /* RVVLA_H */
