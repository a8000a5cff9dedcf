// solver.cu — conjugate gradients over the CRS kernels (no reference
// counterpart: a caller of the SpMV path, for symmetric positive definite A).
//
// One iteration is five launches on the caller's stream and no host
// synchronisation:
//   1. q = A p with the fused dot: the CRS lane-run kernel adds p[row] * v
//      for every row piece v it stores or carries into a per-warp partial,
//      so p^T A p needs no second pass over q;
//   2. one block sums the partials (fixed order) and sets alpha = r.r / p.q;
//   3. x += alpha p, r -= alpha q and per-block partials of the new r.r in
//      the same pass (the axpy/dot epilogue fused);
//   4. one block sums them and sets beta = r.r(new) / r.r(old);
//   5. p = r + beta p.
// The scalars live in device memory; every check_every iterations the host
// reads r.r once to test ||r|| <= rtol ||b||.  All reductions run in a fixed
// order, so a solve is bitwise reproducible.
#include <algorithm>
#include <cmath>
#include <string>
#include <type_traits>

#include "rvvla_internal.cuh"

namespace rvvla {

int crs_spmv_dot_f64(const rvvla_crs* A, const double* p, double* q, double* part, int64_t cap, int64_t* nparts,
                     cudaStream_t st);
int crs_spmv_dot_f32(const rvvla_crs* A, const float* p, float* q, float* part, int64_t cap, int64_t* nparts,
                     cudaStream_t st);
int64_t crs_warp_count(int64_t nz);

namespace {

struct CgScalars {
  double rr;      // r.r of the current residual
  double pq;      // p.(A p)
  double alpha, beta;
  double bb;      // b.b
};

constexpr int kRedThreads = 1024;
constexpr int kUpdThreads = 256;

// Sum of v[0..n) by one block: thread t adds t, t + 1024, ... in order, then
// a fixed tree in shared memory.
template <class T>
__device__ double block_sum(const T* __restrict__ v, int64_t n) {
  __shared__ double sh[kRedThreads];
  double a = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += kRedThreads) a += (double)v[i];
  sh[threadIdx.x] = a;
  __syncthreads();
  for (int d = kRedThreads / 2; d > 0; d >>= 1) {
    if ((int)threadIdx.x < d) sh[threadIdx.x] += sh[threadIdx.x + d];
    __syncthreads();
  }
  return sh[0];
}

template <class T>
__global__ void __launch_bounds__(kRedThreads) cg_alpha_kernel(const T* __restrict__ part, int64_t n, CgScalars* s) {
  const double pq = block_sum(part, n);
  if (threadIdx.x == 0) {
    s->pq = pq;
    s->alpha = pq != 0.0 ? s->rr / pq : 0.0;
  }
}

__global__ void __launch_bounds__(kRedThreads) cg_beta_kernel(const double* __restrict__ part, int64_t n,
                                                              CgScalars* s) {
  const double rr = block_sum(part, n);
  if (threadIdx.x == 0) {
    s->beta = s->rr != 0.0 ? rr / s->rr : 0.0;
    s->rr = rr;
  }
}

// per-block partial of u.v over a grid-stride loop (fixed grid: fixed order)
__device__ void block_partial(double a, double* __restrict__ part) {
  __shared__ double sh[kUpdThreads];
  sh[threadIdx.x] = a;
  __syncthreads();
  for (int d = kUpdThreads / 2; d > 0; d >>= 1) {
    if ((int)threadIdx.x < d) sh[threadIdx.x] += sh[threadIdx.x + d];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

template <class T>
__global__ void __launch_bounds__(kUpdThreads) cg_dot_kernel(int64_t n, const T* __restrict__ u,
                                                             const T* __restrict__ v, double* __restrict__ part) {
  double a = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kUpdThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kUpdThreads)
    a += (double)u[i] * (double)v[i];
  block_partial(a, part);
}

__global__ void __launch_bounds__(kRedThreads) cg_set_kernel(const double* __restrict__ part, int64_t n,
                                                             CgScalars* s, int which) {
  const double v = block_sum(part, n);
  if (threadIdx.x == 0) {
    if (which == 0) s->rr = v;
    else s->bb = v;
  }
}

template <class T>
__global__ void __launch_bounds__(kUpdThreads) cg_update_kernel(int64_t n, T* __restrict__ x, T* __restrict__ r,
                                                                const T* __restrict__ p, const T* __restrict__ q,
                                                                const CgScalars* __restrict__ s,
                                                                double* __restrict__ part) {
  const T alpha = (T)s->alpha;
  double a = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kUpdThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kUpdThreads) {
    x[i] += alpha * p[i];
    const T ri = r[i] - alpha * q[i];
    r[i] = ri;
    a += (double)ri * (double)ri;
  }
  block_partial(a, part);
}

template <class T>
__global__ void __launch_bounds__(kRedThreads) sum_to_kernel(const T* __restrict__ part, int64_t n, T* out) {
  const double v = block_sum(part, n);
  if (threadIdx.x == 0) *out = (T)v;
}

template <class T>
int spmv_dot_impl(const rvvla_crs* A, const T* x, T* y, T* dot, cudaStream_t st) {
  if (!A || !x || !y || !dot) return fail(RVVLA_ERR_INVALID_ARG, "crs_spmv_dot: null argument");
  if (A->m != A->n) return fail(RVVLA_ERR_INVALID_ARG, "crs_spmv_dot: A must be square");
  if (A->m == 0 || A->nz == 0) {  // y = 0, dot = 0
    if (A->m > 0) RVVLA_CUDA(cudaMemsetAsync(y, 0, (size_t)A->m * sizeof(T), st));
    RVVLA_CUDA(cudaMemsetAsync(dot, 0, sizeof(T), st));
    return RVVLA_OK;
  }
  const int64_t nw = crs_warp_count(A->nz);
  Scratch sc;
  RVVLA_CUDA(sc.alloc((size_t)nw * sizeof(T), st));
  int64_t np = 0;
  const int rc = std::is_same<T, double>::value
                     ? crs_spmv_dot_f64(A, reinterpret_cast<const double*>(x), reinterpret_cast<double*>(y),
                                        sc.as<double>(), nw, &np, st)
                     : crs_spmv_dot_f32(A, reinterpret_cast<const float*>(x), reinterpret_cast<float*>(y),
                                        sc.as<float>(), nw, &np, st);
  if (rc) return rc;
  sum_to_kernel<T><<<1, kRedThreads, 0, st>>>(sc.as<T>(), np, dot);
  RVVLA_LAUNCHED("sum_to_kernel");
  return RVVLA_OK;
}

template <class T>
__global__ void cg_p_kernel(int64_t n, T* __restrict__ p, const T* __restrict__ r, const CgScalars* __restrict__ s) {
  const T beta = (T)s->beta;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = r[i] + beta * p[i];
}

template <class T>
int cg_impl(const rvvla_crs* A, const T* b, T* x, int64_t max_iter, double rtol, int64_t check_every, int64_t* iters,
            double* rel_res, cudaStream_t st) {
  if (!A || !b || !x || !iters || !rel_res) return fail(RVVLA_ERR_INVALID_ARG, "cg: null argument");
  if (A->m != A->n || A->m <= 0) return fail(RVVLA_ERR_INVALID_ARG, "cg: A must be square and non-empty");
  if (max_iter < 0 || check_every <= 0 || !(rtol >= 0.0))
    return fail(RVVLA_ERR_INVALID_ARG, "cg: bad iteration limits");
  if (A->nz == 0 || !A->plan || (A->plan_kind != 1 && A->plan_kind != 2))
    return fail(RVVLA_ERR_INVALID_ARG, "cg: A needs nonzeros and an analysed plan (rvvla_crs_analyze)");
  const int64_t n = A->n;
  const int64_t nw = crs_warp_count(A->nz);
  const int upd_blocks = (int)std::min<int64_t>((n + kUpdThreads - 1) / kUpdThreads, (int64_t)sm_count() * 8);
  Scratch sc;
  const size_t vec = ((size_t)n * sizeof(T) + 255) / 256 * 256;
  const size_t partb = ((size_t)std::max<int64_t>(nw, 1) * sizeof(T) + 255) / 256 * 256;
  const size_t rrb = ((size_t)upd_blocks * sizeof(double) + 255) / 256 * 256;
  RVVLA_CUDA(sc.alloc(3 * vec + partb + rrb + sizeof(CgScalars), st));
  char* base = sc.as<char>();
  T* r = reinterpret_cast<T*>(base);
  T* p = reinterpret_cast<T*>(base + vec);
  T* q = reinterpret_cast<T*>(base + 2 * vec);
  T* part = reinterpret_cast<T*>(base + 3 * vec);
  double* rrp = reinterpret_cast<double*>(base + 3 * vec + partb);
  CgScalars* s = reinterpret_cast<CgScalars*>(base + 3 * vec + partb + rrb);
  // r = b - A x, p = r, r.r, b.b
  RVVLA_CUDA(cudaMemcpyAsync(r, b, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, st));
  int rc = std::is_same<T, double>::value
               ? rvvla_crs_spmv_f64(A, -1.0, reinterpret_cast<const double*>(x), 1.0, reinterpret_cast<double*>(r),
                                    (void*)st)
               : rvvla_crs_spmv_f32(A, -1.0f, reinterpret_cast<const float*>(x), 1.0f, reinterpret_cast<float*>(r),
                                    (void*)st);
  if (rc) return rc;
  RVVLA_CUDA(cudaMemcpyAsync(p, r, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, st));
  cg_dot_kernel<T><<<upd_blocks, kUpdThreads, 0, st>>>(n, r, r, rrp);
  RVVLA_LAUNCHED("cg_dot_kernel");
  cg_set_kernel<<<1, kRedThreads, 0, st>>>(rrp, upd_blocks, s, 0);
  RVVLA_LAUNCHED("cg_set_kernel");
  cg_dot_kernel<T><<<upd_blocks, kUpdThreads, 0, st>>>(n, b, b, rrp);
  RVVLA_LAUNCHED("cg_dot_kernel");
  cg_set_kernel<<<1, kRedThreads, 0, st>>>(rrp, upd_blocks, s, 1);
  RVVLA_LAUNCHED("cg_set_kernel");
  CgScalars hs{};
  auto read_back = [&]() -> int {
    RVVLA_CUDA(cudaMemcpyAsync(&hs, s, sizeof(hs), cudaMemcpyDeviceToHost, st));
    RVVLA_CUDA(cudaStreamSynchronize(st));
    return RVVLA_OK;
  };
  if ((rc = read_back())) return rc;
  const double bb = hs.bb > 0.0 ? hs.bb : 1.0;
  int64_t it = 0;
  bool done = std::sqrt(hs.rr / bb) <= rtol;
  while (!done && it < max_iter) {
    int64_t np = 0;
    rc = std::is_same<T, double>::value
             ? crs_spmv_dot_f64(A, reinterpret_cast<const double*>(p), reinterpret_cast<double*>(q),
                                reinterpret_cast<double*>(part), nw, &np, st)
             : crs_spmv_dot_f32(A, reinterpret_cast<const float*>(p), reinterpret_cast<float*>(q),
                                reinterpret_cast<float*>(part), nw, &np, st);
    if (rc) return rc;
    cg_alpha_kernel<T><<<1, kRedThreads, 0, st>>>(part, np, s);
    RVVLA_LAUNCHED("cg_alpha_kernel");
    cg_update_kernel<T><<<upd_blocks, kUpdThreads, 0, st>>>(n, x, r, p, q, s, rrp);
    RVVLA_LAUNCHED("cg_update_kernel");
    cg_beta_kernel<<<1, kRedThreads, 0, st>>>(rrp, upd_blocks, s);
    RVVLA_LAUNCHED("cg_beta_kernel");
    cg_p_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, p, r, s);
    RVVLA_LAUNCHED("cg_p_kernel");
    ++it;
    if (it % check_every == 0 || it == max_iter) {
      if ((rc = read_back())) return rc;
      done = std::sqrt(hs.rr / bb) <= rtol;
    }
  }
  *iters = it;
  *rel_res = std::sqrt(hs.rr / bb);
  return RVVLA_OK;
}

}  // namespace
}  // namespace rvvla

using namespace rvvla;

extern "C" {

int rvvla_cg_f64(const rvvla_crs* A, const double* b, double* x, int64_t max_iter, double rtol, int64_t check_every,
                 int64_t* iters, double* rel_res, void* stream) {
  return cg_impl<double>(A, b, x, max_iter, rtol, check_every, iters, rel_res, as_stream(stream));
}

int rvvla_cg_f32(const rvvla_crs* A, const float* b, float* x, int64_t max_iter, double rtol, int64_t check_every,
                 int64_t* iters, double* rel_res, void* stream) {
  return cg_impl<float>(A, b, x, max_iter, rtol, check_every, iters, rel_res, as_stream(stream));
}

int rvvla_crs_spmv_dot_f64(const rvvla_crs* A, const double* x, double* y, double* dot, void* stream) {
  return spmv_dot_impl<double>(A, x, y, dot, as_stream(stream));
}

int rvvla_crs_spmv_dot_f32(const rvvla_crs* A, const float* x, float* y, float* dot, void* stream) {
  return spmv_dot_impl<float>(A, x, y, dot, as_stream(stream));
}

}  // extern "C"
