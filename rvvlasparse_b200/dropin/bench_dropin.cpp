// bench_dropin.cpp — the end-to-end leg of bench.py: sparse_mv through the
// C++ drop-in exactly as a caller of the reference API makes it, with host
// std::vector b and y (every call copies b to the device and y back), for
// each (format, precision) case of the bench, one after another.
//
//   bench_dropin <powerlaw|stencil|laplace> <n> <formats,...> <precisions,...> <steps> <warmup>
//
// The matrix comes from the library's seeded generators (the same bits as the
// bench's device-resident leg); every format is built by the drop-in's
// convert (on the GPU) with the bench's parameters; the mixed cases call the
// drop-in's sparse_mv_mixed on the float matrix.  Each case's time is the
// median over the timed steps of the host wall time of one call, which
// returns only when y is back in host memory.  Prints one JSON line: per
// case the median ms, and per step the bytes copied each way.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "rvvla.h"
#include "sparse_matrix.h"

using namespace SparseMatrixLib;

namespace {

std::vector<std::string> split(const std::string& s) {
  std::vector<std::string> out;
  size_t a = 0;
  while (a <= s.size()) {
    size_t b = s.find(',', a);
    if (b == std::string::npos) b = s.size();
    if (b > a) out.push_back(s.substr(a, b - a));
    a = b + 1;
  }
  return out;
}

struct Csr {
  int64_t m = 0, n = 0;
  std::vector<int32_t> R, C;
  std::vector<double> V;
};

Csr generate(const std::string& w, int64_t n) {
  Csr a;
  int64_t nz = -1;
  if (w == "powerlaw") {
    a.m = a.n = n;
    nz = rvvla_gen_powerlaw(n, 16.0, 1.2, 4096, 1024, 0.7, 1, nullptr, nullptr, nullptr);
  } else if (w == "stencil") {
    a.m = a.n = 128 * 128 * 128;
    nz = rvvla_gen_stencil27(128, 3, nullptr, nullptr, nullptr);
  } else if (w == "laplace") {
    a.m = a.n = 256 * 256;
    nz = rvvla_gen_laplace2d(256, nullptr, nullptr, nullptr);
  }
  if (nz < 0) throw std::runtime_error("unknown workload " + w);
  a.R.resize((size_t)a.m + 1);
  a.C.resize((size_t)nz);
  a.V.resize((size_t)nz);
  if (w == "powerlaw") rvvla_gen_powerlaw(n, 16.0, 1.2, 4096, 1024, 0.7, 1, a.R.data(), a.C.data(), a.V.data());
  else if (w == "stencil") rvvla_gen_stencil27(128, 3, a.R.data(), a.C.data(), a.V.data());
  else rvvla_gen_laplace2d(256, a.R.data(), a.C.data(), a.V.data());
  return a;
}

// one case: a callable doing one sparse_mv with host vectors
struct Case {
  std::string name;
  std::function<int()> call;
  size_t h2d = 0, d2h = 0;
  std::vector<double> ms;
};

template <class T>
std::unique_ptr<spMtxCRS<T>> crs_of(const Csr& a) {
  std::vector<T> v(a.V.begin(), a.V.end());
  return std::make_unique<spMtxCRS<T>>((size_t)a.m, (size_t)a.n, a.C.size(), a.R.data(), a.C.data(), v.data());
}

convertParams params(std::initializer_list<std::pair<const char*, int>> ints,
                     std::initializer_list<std::pair<const char*, double>> dbls = {}) {
  convertParams cp;
  for (const auto& kv : ints) cp.param[kv.first].i = kv.second;
  for (const auto& kv : dbls) cp.param[kv.first].d = kv.second;
  return cp;
}

// the format built from a CRS with the bench's parameters (held as void)
template <class T>
std::shared_ptr<void> build(const std::string& fmt, spMtxCRS<T>& A, size_t n) {
  if (fmt == "crs") return std::shared_ptr<void>(&A, [](void*) {});
  if (fmt == "hcsr") {
    auto p = std::make_shared<spMtxHCSR<T>>();
    convert(*p, A, convertParams{});
    return p;
  }
  if (fmt == "csr5") {
    auto p = std::make_shared<spMtxCSR5<T>>();
    convert(*p, A, params({{"omega", 32}, {"sigma", 16}}));
    return p;
  }
  if (fmt == "sell") {
    auto p = std::make_shared<spMtxSELL_C_Sigma<T>>();
    convert(*p, A, params({{"C", 32}, {"Sigma", 256}}));
    return p;
  }
  if (fmt == "lav") {
    auto p = std::make_shared<spMtxLAV<T>>();
    convert(*p, A, params({{"SIMD_Lanes", 8}, {"segment_len", (int)std::max<size_t>(n, 1)}}, {{"T", 0.2}}));
    return p;
  }
  if (fmt == "vnec") return std::make_shared<spMtxVNEC<T>>(A);
  if (fmt == "vhcc") {
    auto p = std::make_shared<spMtxVHCC<T>>();
    convert(*p, A, convertParams{});
    return p;
  }
  if (fmt == "cvr") {
    auto p = std::make_shared<spMtxCVR<T>>();
    convert(*p, A, convertParams{});
    return p;
  }
  throw std::runtime_error("unknown format " + fmt);
}

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 7) {
    std::fprintf(stderr, "usage: %s workload n formats precisions steps warmup\n", argv[0]);
    return 2;
  }
  const std::string wl = argv[1];
  const int64_t n_arg = std::atoll(argv[2]);
  const auto formats = split(argv[3]), precs = split(argv[4]);
  const int steps = std::max(1, std::atoi(argv[5])), warmup = std::max(1, std::atoi(argv[6]));
  try {
    const Csr a = generate(wl, n_arg);
    const size_t m = (size_t)a.m, n = (size_t)a.n;
    auto A64 = crs_of<double>(a);
    auto A32 = crs_of<float>(a);
    std::vector<double> x64(n), y64(m);
    std::vector<float> x32(n), y32(m);
    rvvla_gen_vector((int64_t)n, 0, 0, -1.0, 1.0, x64.data());
    for (size_t i = 0; i < n; ++i) x32[i] = (float)x64[i];
    std::vector<std::shared_ptr<void>> keep;  // built matrices
    std::vector<Case> cases;
    auto add = [&](const std::string& name, std::function<int()> f, size_t vb) {
      Case c;
      c.name = name;
      c.call = std::move(f);
      c.h2d = n * vb;
      c.d2h = m * vb;
      cases.push_back(std::move(c));
    };
    const sparse_matrix_descr descr{};
    const auto NT = SPARSE_OPERATION_NON_TRANSPOSE;
    for (const auto& fmt : formats) {
      const bool mixable = fmt == "crs" || fmt == "hcsr" || fmt == "csr5" || fmt == "sell";
      std::shared_ptr<void> M64, M32;
      for (const auto& pr : precs) {
        if (pr.rfind("mixed", 0) == 0 && (!mixable || pr != "mixed")) continue;
        const std::string name = fmt + "_" + pr;
        if (pr == "f64") {
          if (!M64) M64 = build<double>(fmt, *A64, n);
          void* raw = M64.get();
#define CASE64(CLS)                                                                                     \
  add(name, [&, raw] {                                                                                  \
    return sparse_mv<double, CLS>(NT, 1.0, *static_cast<CLS<double>*>(raw), descr, x64, 0.0, y64).code; \
  }, 8)
          if (fmt == "crs") CASE64(spMtxCRS);
          else if (fmt == "hcsr") CASE64(spMtxHCSR);
          else if (fmt == "csr5") CASE64(spMtxCSR5);
          else if (fmt == "sell") CASE64(spMtxSELL_C_Sigma);
          else if (fmt == "lav") CASE64(spMtxLAV);
          else if (fmt == "vnec") CASE64(spMtxVNEC);
          else if (fmt == "vhcc") CASE64(spMtxVHCC);
          else if (fmt == "cvr") CASE64(spMtxCVR);
#undef CASE64
        } else {
          if (!M32) M32 = build<float>(fmt, *A32, n);
          void* raw = M32.get();
          const bool mixed = pr == "mixed";
#define CASE32(CLS)                                                                        \
  add(name, [&, raw, mixed] {                                                              \
    const auto& M = *static_cast<CLS<float>*>(raw);                                        \
    return mixed ? sparse_mv_mixed<CLS>(NT, 1.0f, M, descr, x32, 0.0f, y32).code         \
                 : sparse_mv<float, CLS>(NT, 1.0f, M, descr, x32, 0.0f, y32).code;         \
  }, 4)
#define CASE32_PLAIN(CLS)                                                                       \
  add(name, [&, raw] {                                                                          \
    return sparse_mv<float, CLS>(NT, 1.0f, *static_cast<CLS<float>*>(raw), descr, x32, 0.0f, y32).code; \
  }, 4)
          if (fmt == "crs") CASE32(spMtxCRS);
          else if (fmt == "hcsr") CASE32(spMtxHCSR);
          else if (fmt == "csr5") CASE32(spMtxCSR5);
          else if (fmt == "sell") CASE32(spMtxSELL_C_Sigma);
          else if (fmt == "lav") CASE32_PLAIN(spMtxLAV);
          else if (fmt == "vnec") CASE32_PLAIN(spMtxVNEC);
          else if (fmt == "vhcc") CASE32_PLAIN(spMtxVHCC);
          else if (fmt == "cvr") CASE32_PLAIN(spMtxCVR);
#undef CASE32
#undef CASE32_PLAIN
        }
      }
      keep.push_back(M64);
      keep.push_back(M32);
    }
    for (int w = 0; w < warmup; ++w)
      for (auto& c : cases) {
        const int rc = c.call();
        if (rc) throw std::runtime_error(c.name + ": status " + std::to_string(rc) + ": " + rvvla_last_error());
      }
    for (int s = 0; s < steps; ++s)
      for (auto& c : cases) {
        const double t0 = now_ms();
        const int rc = c.call();
        const double t1 = now_ms();
        if (rc) throw std::runtime_error(c.name + ": status " + std::to_string(rc));
        c.ms.push_back(t1 - t0);
      }
    size_t h2d = 0, d2h = 0;
    std::printf("{\"cases\": {");
    for (size_t i = 0; i < cases.size(); ++i) {
      auto v = cases[i].ms;
      std::sort(v.begin(), v.end());
      const double med = v[v.size() / 2];
      h2d += cases[i].h2d;
      d2h += cases[i].d2h;
      std::printf("%s\"%s\": {\"ms\": %.6f}", i ? ", " : "", cases[i].name.c_str(), med);
    }
    std::printf("}, \"h2d_bytes_per_step\": %zu, \"d2h_bytes_per_step\": %zu, \"m\": %zu, \"n\": %zu, \"nnz\": %zu}\n",
                h2d, d2h, m, n, a.C.size());
  } catch (const std::exception& e) {
    std::fprintf(stderr, "bench_dropin: %s\n", e.what());
    return 1;
  }
  return 0;
}
