// autotune.cu — measuring autotuner for the single-matrix formats, in the C
// ABI so that C++ callers of the drop-in get tuned convertParams
// (include/convert.h:21-28 of the reference is the parameter bag it fills).
//
// For every candidate parameter set the format is built on the GPU from the
// caller's CRS, one product is run untimed, then `iters` products are timed
// with CUDA events on `stream` and the best time kept; the build is freed
// before the next candidate.  Candidates per format:
//   HCSR   square blocks R = C in {512, 1024, 2000, 4000, 8192},
//          R in {1000, 2000, 4000} with C = 65536, and C = 65536 with R
//          making b_m 2, 3 or 4 waves of two CTAs per SM, p = 2;
//   SELL   C = 32 (a warp per slice), sigma in {32, 256, 1024, 8192};
//   CSR5   omega = 32, sigma in {8, 16, 24, 32};
//   LAV    SIMD_Lanes 8, T 0.2, segment_len in {40000, n/4, n};
//   VHCC   num_threads in {nnz/4096, nnz/2048, nnz/1024};
//   CVR    Nthreads in {nnz/8192, nnz/32768, nnz/131072}.
// x and y are scratch vectors of the library (the timing does not depend on
// their values).
#include <algorithm>
#include <vector>

#include "rvvla_internal.cuh"

namespace rvvla {
namespace {

std::vector<rvvla_tune_params> candidates(int fmt, const rvvla_crs* A) {
  std::vector<rvvla_tune_params> out;
  auto blank = [] {
    rvvla_tune_params p{};
    p.p = 2.0;
    p.T = 0.2;
    p.simd_lanes = 8;
    return p;
  };
  switch (fmt) {
    case RVVLA_FMT_HCSR:
      for (int64_t b : {512, 1024, 2000, 4000, 8192}) {
        auto p = blank();
        p.R = p.C = b;
        out.push_back(p);
      }
      // the widest blocks the uint16 columns allow: fewer, larger blocks
      for (int64_t r : {1000, 2000, 4000}) {
        auto p = blank();
        p.R = r;
        p.C = 65536;
        out.push_back(p);
      }
      // block rows in whole waves: the kernel runs a CTA per block row, two
      // per SM, so b_m a multiple of 2 x SMs leaves no partial last wave
      for (int64_t waves : {2, 3, 4}) {
        const int64_t slots = 2 * (int64_t)sm_count() * waves;
        auto p = blank();
        p.R = std::max<int64_t>(1, (A->m + slots - 1) / slots);
        p.C = 65536;
        out.push_back(p);
      }
      break;
    case RVVLA_FMT_SELL:
      for (int64_t s : {32, 256, 1024, 8192}) {
        auto p = blank();
        p.C = 32;
        p.sigma = s;
        out.push_back(p);
      }
      break;
    case RVVLA_FMT_CSR5:
      for (int64_t s : {8, 16, 24, 32}) {
        auto p = blank();
        p.sigma = s;
        out.push_back(p);
      }
      break;
    case RVVLA_FMT_LAV: {
      std::vector<int64_t> sl = {40000, std::max<int64_t>(1, A->n / 4), std::max<int64_t>(1, A->n)};
      std::sort(sl.begin(), sl.end());
      sl.erase(std::unique(sl.begin(), sl.end()), sl.end());
      for (int64_t s : sl) {
        auto p = blank();
        p.segment_len = s;
        out.push_back(p);
      }
      break;
    }
    case RVVLA_FMT_VHCC:
      for (int64_t d : {4096, 2048, 1024}) {
        auto p = blank();
        p.threads = std::max<int64_t>(1, A->nz / d);
        out.push_back(p);
      }
      break;
    case RVVLA_FMT_CVR:
      for (int64_t d : {8192, 32768, 131072}) {
        auto p = blank();
        p.threads = std::max<int64_t>(1, A->nz / d);
        out.push_back(p);
      }
      break;
    default:
      break;
  }
  return out;
}

// one candidate's build, freed with its format's free function
struct Built {
  int fmt = 0;
  rvvla_hcsr_owned h{};
  rvvla_sell_owned s{};
  rvvla_csr5_owned c{};
  rvvla_lav_owned l{};
  rvvla_vhcc_owned v{};
  rvvla_cvr_owned r{};
  ~Built() {
    switch (fmt) {
      case RVVLA_FMT_HCSR: rvvla_hcsr_free(&h); break;
      case RVVLA_FMT_SELL: rvvla_sell_free(&s); break;
      case RVVLA_FMT_CSR5: rvvla_csr5_free(&c); break;
      case RVVLA_FMT_LAV: rvvla_lav_free(&l); break;
      case RVVLA_FMT_VHCC: rvvla_vhcc_free(&v); break;
      case RVVLA_FMT_CVR: rvvla_cvr_free(&r); break;
      default: break;
    }
  }
};

int build(int fmt, const rvvla_crs* A, int vb, const rvvla_tune_params& p, Built& b, cudaStream_t st) {
  void* s = st;
  b.fmt = fmt;
  switch (fmt) {
    case RVVLA_FMT_HCSR: return rvvla_hcsr_build(A, vb, p.R, p.C, p.p, &b.h, s);
    case RVVLA_FMT_SELL: return rvvla_sell_build(A, vb, p.C, p.sigma, &b.s, s);
    case RVVLA_FMT_CSR5: return rvvla_csr5_build(A, vb, 32, (int)p.sigma, &b.c, s);
    case RVVLA_FMT_LAV: return rvvla_lav_build(A, vb, p.simd_lanes, p.T, p.segment_len, &b.l, s);
    case RVVLA_FMT_VHCC: return rvvla_vhcc_build(A, vb, p.threads, &b.v, s);
    case RVVLA_FMT_CVR: return rvvla_cvr_build(A, vb, p.threads, &b.r, s);
    default: b.fmt = 0; return fail(RVVLA_ERR_INVALID_ARG, "rvvla_autotune: unknown format");
  }
}

// one product of a built structure: f64 / f32 / mixed by (vt, mixed)
int run(const Built& b, int vt, int mixed, void* x, void* y, cudaStream_t st) {
  void* s = st;
  const bool f64 = vt == RVVLA_F64;
  const double* xd = static_cast<const double*>(x);
  double* yd = static_cast<double*>(y);
  const float* xf = static_cast<const float*>(x);
  float* yf = static_cast<float*>(y);
  switch (b.fmt) {
    case RVVLA_FMT_HCSR:
      if (mixed) return rvvla_hcsr_spmv_mixed(&b.h.h, vt, 1.f, xf, 0.f, yf, s);
      return f64 ? rvvla_hcsr_spmv_f64(&b.h.h, 1.0, xd, 0.0, yd, s) : rvvla_hcsr_spmv_f32(&b.h.h, 1.f, xf, 0.f, yf, s);
    case RVVLA_FMT_SELL:
      if (mixed) return rvvla_sell_spmv_mixed(&b.s.h, vt, 1.f, xf, 0.f, yf, s);
      return f64 ? rvvla_sell_spmv_f64(&b.s.h, RVVLA_STAGE_ALL, 1.0, xd, 0.0, yd, s)
                 : rvvla_sell_spmv_f32(&b.s.h, RVVLA_STAGE_ALL, 1.f, xf, 0.f, yf, s);
    case RVVLA_FMT_CSR5:
      if (mixed) return rvvla_csr5_spmv_mixed(&b.c.h, vt, 1.f, xf, 0.f, yf, s);
      return f64 ? rvvla_csr5_spmv_f64(&b.c.h, 1.0, xd, 0.0, yd, s) : rvvla_csr5_spmv_f32(&b.c.h, 1.f, xf, 0.f, yf, s);
    case RVVLA_FMT_LAV:
      return f64 ? rvvla_lav_spmv_f64(&b.l.h, 1.0, xd, 0.0, yd, s) : rvvla_lav_spmv_f32(&b.l.h, 1.f, xf, 0.f, yf, s);
    case RVVLA_FMT_VHCC:
      return f64 ? rvvla_vhcc_spmv_f64(&b.v.h, 1.0, xd, 0.0, yd, s) : rvvla_vhcc_spmv_f32(&b.v.h, 1.f, xf, 0.f, yf, s);
    case RVVLA_FMT_CVR:
      return f64 ? rvvla_cvr_spmv_f64(&b.r.h, 1.0, xd, 0.0, yd, s) : rvvla_cvr_spmv_f32(&b.r.h, 1.f, xf, 0.f, yf, s);
    default:
      return fail(RVVLA_ERR_INVALID_ARG, "rvvla_autotune: unknown format");
  }
}

struct Events {
  cudaEvent_t a = nullptr, b = nullptr;
  ~Events() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

}  // namespace
}  // namespace rvvla

using namespace rvvla;

extern "C" int rvvla_autotune(int format, const rvvla_crs* src, int val_type, int mixed, int iters,
                              rvvla_tune_params* best, double* best_ms, rvvla_tune_params* table, double* table_ms,
                              int table_cap, int* n_candidates, void* stream) {
  if (!src || !best) return fail(RVVLA_ERR_INVALID_ARG, "rvvla_autotune: null argument");
  if (val_type != RVVLA_F64 && val_type != RVVLA_F32 && val_type != RVVLA_BF16)
    return fail(RVVLA_ERR_INVALID_ARG, "rvvla_autotune: val_type must be RVVLA_F64, RVVLA_F32 or RVVLA_BF16");
  const bool mixable = format == RVVLA_FMT_HCSR || format == RVVLA_FMT_SELL || format == RVVLA_FMT_CSR5;
  if (mixed && (!mixable || val_type == RVVLA_F64))
    return fail(RVVLA_ERR_INVALID_ARG,
                "rvvla_autotune: the mixed form exists for HCSR, SELL and CSR5 with F32 or BF16 values");
  if (!mixed && val_type == RVVLA_BF16)
    return fail(RVVLA_ERR_INVALID_ARG, "rvvla_autotune: BF16 values only in the mixed form");
  if (src->m <= 0 || src->n <= 0 || src->nz <= 0) return fail(RVVLA_ERR_INVALID_ARG, "rvvla_autotune: empty matrix");
  const auto cands = candidates(format, src);
  if (cands.empty()) return fail(RVVLA_ERR_INVALID_ARG, "rvvla_autotune: unknown format");
  if (n_candidates) *n_candidates = (int)cands.size();
  iters = std::max(1, iters);
  cudaStream_t st = as_stream(stream);
  const int vb = val_type == RVVLA_F64 ? 8 : val_type == RVVLA_F32 ? 4 : 2;
  const size_t xb = val_type == RVVLA_F64 ? 8 : 4;
  Scratch sx, sy;
  RVVLA_CUDA(sx.alloc((size_t)src->n * xb, st));
  RVVLA_CUDA(sy.alloc((size_t)src->m * xb, st));
  RVVLA_CUDA(cudaMemsetAsync(sx.p, 0, (size_t)src->n * xb, st));
  Events ev;
  RVVLA_CUDA(cudaEventCreate(&ev.a));
  RVVLA_CUDA(cudaEventCreate(&ev.b));
  double bestv = -1.0;
  for (size_t i = 0; i < cands.size(); ++i) {
    Built b;
    int rc = build(format, src, vb, cands[i], b, st);
    if (rc) return rc;
    if ((rc = run(b, val_type, mixed, sx.p, sy.p, st))) return rc;  // untimed
    float ms = 1e30f;
    for (int it = 0; it < iters; ++it) {
      RVVLA_CUDA(cudaEventRecord(ev.a, st));
      if ((rc = run(b, val_type, mixed, sx.p, sy.p, st))) return rc;
      RVVLA_CUDA(cudaEventRecord(ev.b, st));
      RVVLA_CUDA(cudaEventSynchronize(ev.b));
      float t = 0.f;
      RVVLA_CUDA(cudaEventElapsedTime(&t, ev.a, ev.b));
      ms = std::min(ms, t);
    }
    if (table && (int)i < table_cap) table[i] = cands[i];
    if (table_ms && (int)i < table_cap) table_ms[i] = ms;
    if (bestv < 0 || ms < bestv) {
      bestv = ms;
      *best = cands[i];
    }
  }
  if (best_ms) *best_ms = bestv;
  RVVLA_CUDA(cudaStreamSynchronize(st));
  return RVVLA_OK;
}
