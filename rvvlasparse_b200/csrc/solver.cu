// solver.cu — conjugate gradients (symmetric positive definite A) and
// BiCGStab (general square A) over the CRS kernels (no reference
// counterpart: callers of the SpMV path).
//
// A CG iteration is five launches on the caller's stream and no host
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

// ---------------------------------------------------------------- BiCGStab
// Unpreconditioned BiCGStab (van der Vorst 1992) for a general square A, on
// the same pieces: per iteration two CRS products (v = A p, t = A s), the
// dots r^.v, t.s, t.t, r^.r and r.r as per-block partials summed by one
// block in a fixed order, and three fused vector passes.  Scalars stay on
// the device; the host reads them every check_every iterations.
struct BiScalars {
  double rho;    // r^.r of the current residual
  double alpha, omega, beta;
  double rr;     // r.r
  double bb;     // b.b
  int breakdown;  // rho, r^.v or t.t became exactly zero
};

template <class T>
__global__ void __launch_bounds__(kUpdThreads) bi_p_kernel(int64_t n, T* __restrict__ p, const T* __restrict__ r,
                                                           const T* __restrict__ v, const BiScalars* __restrict__ s) {
  const T beta = (T)s->beta, omega = (T)s->omega;
  for (int64_t i = (int64_t)blockIdx.x * kUpdThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kUpdThreads)
    p[i] = r[i] + beta * (p[i] - omega * v[i]);
}

__global__ void __launch_bounds__(kRedThreads) bi_alpha_kernel(const double* __restrict__ part, int64_t np,
                                                               BiScalars* s) {
  const double rv = block_sum(part, np);
  if (threadIdx.x == 0) {
    s->alpha = rv != 0.0 ? s->rho / rv : 0.0;
    if (rv == 0.0) s->breakdown = 1;
  }
}

template <class T>
__global__ void __launch_bounds__(kUpdThreads) bi_s_kernel(int64_t n, T* __restrict__ sv, const T* __restrict__ r,
                                                           const T* __restrict__ v, const BiScalars* __restrict__ s) {
  const T alpha = (T)s->alpha;
  for (int64_t i = (int64_t)blockIdx.x * kUpdThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kUpdThreads)
    sv[i] = r[i] - alpha * v[i];
}

// partials of u1.v1 and u2.v2 in one pass
template <class T>
__global__ void __launch_bounds__(kUpdThreads) dot2_kernel(int64_t n, const T* __restrict__ u1, const T* __restrict__ v1,
                                                           const T* __restrict__ u2, const T* __restrict__ v2,
                                                           double* __restrict__ part1, double* __restrict__ part2) {
  double a = 0.0, b = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kUpdThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kUpdThreads) {
    a += (double)u1[i] * (double)v1[i];
    b += (double)u2[i] * (double)v2[i];
  }
  block_partial(a, part1);
  block_partial(b, part2);
}

__global__ void __launch_bounds__(kRedThreads) bi_omega_kernel(const double* __restrict__ part1,
                                                               const double* __restrict__ part2, int64_t np,
                                                               BiScalars* s) {
  const double ts = block_sum(part1, np);
  __syncthreads();  // every thread has read the first sum before the second reuses the buffer
  const double tt = block_sum(part2, np);
  if (threadIdx.x == 0) {
    s->omega = tt != 0.0 ? ts / tt : 0.0;
    if (tt == 0.0) s->breakdown = 1;
  }
}

// x += alpha p + omega s, r = s - omega t, partials of r^.r and r.r
template <class T>
__global__ void __launch_bounds__(kUpdThreads) bi_xr_kernel(int64_t n, T* __restrict__ x, T* __restrict__ r,
                                                            const T* __restrict__ p, const T* __restrict__ sv,
                                                            const T* __restrict__ t, const T* __restrict__ rh,
                                                            const BiScalars* __restrict__ s, double* __restrict__ part1,
                                                            double* __restrict__ part2) {
  const T alpha = (T)s->alpha, omega = (T)s->omega;
  double a = 0.0, b = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kUpdThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kUpdThreads) {
    x[i] += alpha * p[i] + omega * sv[i];
    const T ri = sv[i] - omega * t[i];
    r[i] = ri;
    a += (double)rh[i] * (double)ri;
    b += (double)ri * (double)ri;
  }
  block_partial(a, part1);
  block_partial(b, part2);
}

__global__ void __launch_bounds__(kRedThreads) bi_rho_kernel(const double* __restrict__ part1,
                                                             const double* __restrict__ part2, int64_t np,
                                                             BiScalars* s, int init) {
  const double rho = block_sum(part1, np);
  __syncthreads();  // as above
  const double rr = block_sum(part2, np);
  if (threadIdx.x == 0) {
    if (init) {
      s->beta = 0.0;
      s->omega = 1.0;
      s->alpha = 1.0;
      s->breakdown = 0;
    } else {
      const bool ok = s->rho != 0.0 && s->omega != 0.0;
      s->beta = ok ? (rho / s->rho) * (s->alpha / s->omega) : 0.0;
      if (!ok || rho == 0.0) s->breakdown = 1;
    }
    s->rho = rho;
    s->rr = rr;
  }
}

template <class T>
int crs_product(const rvvla_crs* A, const T* x, T* y, cudaStream_t st) {
  return std::is_same<T, double>::value
             ? rvvla_crs_spmv_f64(A, 1.0, reinterpret_cast<const double*>(x), 0.0, reinterpret_cast<double*>(y),
                                  (void*)st)
             : rvvla_crs_spmv_f32(A, 1.0f, reinterpret_cast<const float*>(x), 0.0f, reinterpret_cast<float*>(y),
                                  (void*)st);
}

template <class T>
int bicgstab_impl(const rvvla_crs* A, const T* b, T* x, int64_t max_iter, double rtol, int64_t check_every,
                  int64_t* iters, double* rel_res, int* breakdown, cudaStream_t st) {
  if (!A || !b || !x || !iters || !rel_res || !breakdown) return fail(RVVLA_ERR_INVALID_ARG, "bicgstab: null argument");
  if (A->m != A->n || A->m <= 0) return fail(RVVLA_ERR_INVALID_ARG, "bicgstab: A must be square and non-empty");
  if (max_iter < 0 || check_every <= 0 || !(rtol >= 0.0))
    return fail(RVVLA_ERR_INVALID_ARG, "bicgstab: bad iteration limits");
  if (A->nz == 0 || !A->plan || (A->plan_kind != 1 && A->plan_kind != 2))
    return fail(RVVLA_ERR_INVALID_ARG, "bicgstab: A needs nonzeros and an analysed plan (rvvla_crs_analyze)");
  const int64_t n = A->n;
  const int upd_blocks = (int)std::min<int64_t>((n + kUpdThreads - 1) / kUpdThreads, (int64_t)sm_count() * 8);
  Scratch sc;
  const size_t vec = ((size_t)n * sizeof(T) + 255) / 256 * 256;
  const size_t pb = ((size_t)upd_blocks * sizeof(double) + 255) / 256 * 256;
  RVVLA_CUDA(sc.alloc(6 * vec + 2 * pb + sizeof(BiScalars), st));
  char* base = sc.as<char>();
  T* r = reinterpret_cast<T*>(base);
  T* rh = reinterpret_cast<T*>(base + vec);
  T* p = reinterpret_cast<T*>(base + 2 * vec);
  T* v = reinterpret_cast<T*>(base + 3 * vec);
  T* sv = reinterpret_cast<T*>(base + 4 * vec);
  T* t = reinterpret_cast<T*>(base + 5 * vec);
  double* part1 = reinterpret_cast<double*>(base + 6 * vec);
  double* part2 = reinterpret_cast<double*>(base + 6 * vec + pb);
  BiScalars* s = reinterpret_cast<BiScalars*>(base + 6 * vec + 2 * pb);
  // r = b - A x, r^ = r, p = v = 0, rho = r^.r, b.b
  RVVLA_CUDA(cudaMemcpyAsync(r, b, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, st));
  int rc = std::is_same<T, double>::value
               ? rvvla_crs_spmv_f64(A, -1.0, reinterpret_cast<const double*>(x), 1.0, reinterpret_cast<double*>(r),
                                    (void*)st)
               : rvvla_crs_spmv_f32(A, -1.0f, reinterpret_cast<const float*>(x), 1.0f, reinterpret_cast<float*>(r),
                                    (void*)st);
  if (rc) return rc;
  RVVLA_CUDA(cudaMemcpyAsync(rh, r, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, st));
  RVVLA_CUDA(cudaMemsetAsync(p, 0, 2 * vec, st));  // p and v
  dot2_kernel<T><<<upd_blocks, kUpdThreads, 0, st>>>(n, rh, r, r, r, part1, part2);
  RVVLA_LAUNCHED("dot2_kernel");
  bi_rho_kernel<<<1, kRedThreads, 0, st>>>(part1, part2, upd_blocks, s, 1);
  RVVLA_LAUNCHED("bi_rho_kernel");
  cg_dot_kernel<T><<<upd_blocks, kUpdThreads, 0, st>>>(n, b, b, part1);
  RVVLA_LAUNCHED("cg_dot_kernel");
  sum_to_kernel<double><<<1, kRedThreads, 0, st>>>(part1, upd_blocks, &s->bb);
  RVVLA_LAUNCHED("sum_to_kernel");
  BiScalars hs{};
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
    bi_p_kernel<T><<<upd_blocks, kUpdThreads, 0, st>>>(n, p, r, v, s);
    RVVLA_LAUNCHED("bi_p_kernel");
    if ((rc = crs_product<T>(A, p, v, st))) return rc;
    cg_dot_kernel<T><<<upd_blocks, kUpdThreads, 0, st>>>(n, rh, v, part1);
    RVVLA_LAUNCHED("cg_dot_kernel");
    bi_alpha_kernel<<<1, kRedThreads, 0, st>>>(part1, upd_blocks, s);
    RVVLA_LAUNCHED("bi_alpha_kernel");
    bi_s_kernel<T><<<upd_blocks, kUpdThreads, 0, st>>>(n, sv, r, v, s);
    RVVLA_LAUNCHED("bi_s_kernel");
    if ((rc = crs_product<T>(A, sv, t, st))) return rc;
    dot2_kernel<T><<<upd_blocks, kUpdThreads, 0, st>>>(n, t, sv, t, t, part1, part2);
    RVVLA_LAUNCHED("dot2_kernel");
    bi_omega_kernel<<<1, kRedThreads, 0, st>>>(part1, part2, upd_blocks, s);
    RVVLA_LAUNCHED("bi_omega_kernel");
    bi_xr_kernel<T><<<upd_blocks, kUpdThreads, 0, st>>>(n, x, r, p, sv, t, rh, s, part1, part2);
    RVVLA_LAUNCHED("bi_xr_kernel");
    bi_rho_kernel<<<1, kRedThreads, 0, st>>>(part1, part2, upd_blocks, s, 0);
    RVVLA_LAUNCHED("bi_rho_kernel");
    ++it;
    if (it % check_every == 0 || it == max_iter) {
      if ((rc = read_back())) return rc;
      done = std::sqrt(hs.rr / bb) <= rtol || hs.breakdown;
    }
  }
  *iters = it;
  *rel_res = std::sqrt(hs.rr / bb);
  *breakdown = hs.breakdown && !(std::sqrt(hs.rr / bb) <= rtol);
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

int rvvla_bicgstab_f64(const rvvla_crs* A, const double* b, double* x, int64_t max_iter, double rtol,
                       int64_t check_every, int64_t* iters, double* rel_res, int* breakdown, void* stream) {
  return bicgstab_impl<double>(A, b, x, max_iter, rtol, check_every, iters, rel_res, breakdown, as_stream(stream));
}

int rvvla_bicgstab_f32(const rvvla_crs* A, const float* b, float* x, int64_t max_iter, double rtol,
                       int64_t check_every, int64_t* iters, double* rel_res, int* breakdown, void* stream) {
  return bicgstab_impl<float>(A, b, x, max_iter, rtol, check_every, iters, rel_res, breakdown, as_stream(stream));
}

int rvvla_crs_spmv_dot_f64(const rvvla_crs* A, const double* x, double* y, double* dot, void* stream) {
  return spmv_dot_impl<double>(A, x, y, dot, as_stream(stream));
}

int rvvla_crs_spmv_dot_f32(const rvvla_crs* A, const float* x, float* y, float* dot, void* stream) {
  return spmv_dot_impl<float>(A, x, y, dot, as_stream(stream));
}

}  // extern "C"
