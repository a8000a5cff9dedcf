// csr5_noalloc.cu — fp64 CSR5 SpMV whose calibrator scratch lives in static
// device storage, so the call allocates no device memory.
//
// The ordinary entry (rvvla_csr5_spmv_f64) takes its calibrator — one value
// and one row index per warp, for rows that cross a warp's tile range — from
// the stream-ordered pool on every call.  Some callers cannot allow that: an
// iterative solver that sizes its Krylov workspaces to fill the device's
// memory up front has nothing left for a pool to grow into, and a time-
// stepping loop that must not meet an out-of-memory error (or a pool-growth
// stall) in the middle of a step cannot let the operator it calls allocate.
// This entry serves them: the scratch is a file-scope __device__ array sized
// for the largest launch the kernel makes on a B200 (48 warps per SM x 148
// SMs = 7104 warps), rounded up to 8192 slots (96 KB).
//
// Set-up: the first call on each device (with that device current) resolves
// the arrays' device addresses with cudaGetSymbolAddress and caches them;
// that first call may load this module's device code, so make it before any
// stream capture begins.  Nothing in the scratch needs to start at zero:
// every warp of the SpMV kernel writes its own slot before the calibration
// kernel, later on the same stream, reads it.  Calls that overlap in time
// (other streams, other host threads, same device) share the one scratch and
// race; serialise them.
#include <mutex>

#include "rvvla_internal.cuh"

namespace rvvla {

template <class V, class X, class Ac, class CT>
int csr5_spmv_dispatch(const rvvla_csr5* A, X alpha, const X* x, X beta, X* y, cudaStream_t st, CT* cal,
                       int* cal_row, int64_t cap, int* status_word, bool regs_only);
int64_t csr5_calibrator_len(const rvvla_csr5* A);

namespace {

constexpr int64_t kNoAllocCalSlots = 8192;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_cal[kNoAllocCalSlots];
static __device__ __align__(256) int g_noalloc_cal_row[kNoAllocCalSlots];
// Status word handed to the kernel; the register-staged kernel used here
// never waits, so it stays at its load-time zero.
static __device__ __align__(256) int g_noalloc_status;

struct NoAllocScratch {
  double* cal = nullptr;
  int* cal_row = nullptr;
  int* status = nullptr;
};

std::mutex g_noalloc_mu;
NoAllocScratch g_noalloc[kNoAllocMaxDevices];

int noalloc_scratch(NoAllocScratch* out) {
  int dev = 0;
  RVVLA_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return fail(RVVLA_ERR_UNSUPPORTED, "csr5_spmv_f64_noalloc: device ordinal beyond 63");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoAllocScratch& s = g_noalloc[dev];
  if (!s.cal) {
    void *cal = nullptr, *row = nullptr, *status = nullptr;
    RVVLA_CUDA(cudaGetSymbolAddress(&cal, g_noalloc_cal));
    RVVLA_CUDA(cudaGetSymbolAddress(&row, g_noalloc_cal_row));
    RVVLA_CUDA(cudaGetSymbolAddress(&status, g_noalloc_status));
    s.cal = static_cast<double*>(cal);
    s.cal_row = static_cast<int*>(row);
    s.status = static_cast<int*>(status);
  }
  *out = s;
  return RVVLA_OK;
}

}  // namespace
}  // namespace rvvla

using namespace rvvla;

extern "C" int rvvla_csr5_spmv_f64_noalloc(const rvvla_csr5* A, double alpha, const double* x, double beta,
                                           double* y, void* stream) {
  if (!A) return fail(RVVLA_ERR_INVALID_ARG, "csr5_spmv_f64_noalloc: null descriptor");
  const int64_t need = csr5_calibrator_len(A);
  if (need > kNoAllocCalSlots)
    return fail(RVVLA_ERR_TOO_LARGE, "csr5_spmv_f64_noalloc: the launch needs " + std::to_string(need) +
                                         " calibrator slots; the static scratch holds 8192");
  NoAllocScratch s;
  const int rc = noalloc_scratch(&s);
  if (rc) return rc;
  return csr5_spmv_dispatch<double, double, double, double>(A, alpha, x, beta, y, as_stream(stream), s.cal,
                                                            s.cal_row, kNoAllocCalSlots, s.status, true);
}
