// test_dropin.cpp — a program written against the RVVLASparse C++ API only
// (sparse_matrix.h, sparse_mv, convert, the spMtx* classes), linked with the
// GPU drop-in.  For every format and both value types it converts a matrix,
// multiplies, and compares with a long-double CSR product computed here.
// With an output path argument it also writes the HCSR arrays built for the
// fp64 Laplacian (defaults R = C = 2000, p = 2) so a test can compare them
// with the reference's own convert<double, spMtxHCSR, false>.
// Exit status 0 when every check passes.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <random>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "sparse_matrix.h"

using namespace SparseMatrixLib;

namespace {

int failures = 0;

void expect(bool ok, const std::string& what) {
  if (!ok) {
    ++failures;
    std::printf("FAIL %s\n", what.c_str());
  }
}

template <class T>
spMtxCRS<T> laplace(int g) {
  const size_t m = (size_t)g * g;
  std::vector<int> R(1, 0), C;
  std::vector<T> V;
  for (int i = 0; i < g; ++i)
    for (int j = 0; j < g; ++j) {
      const int r = i * g + j;
      if (i > 0) { C.push_back(r - g); V.push_back(T(-1)); }
      if (j > 0) { C.push_back(r - 1); V.push_back(T(-1)); }
      C.push_back(r); V.push_back(T(4));
      if (j < g - 1) { C.push_back(r + 1); V.push_back(T(-1)); }
      if (i < g - 1) { C.push_back(r + g); V.push_back(T(-1)); }
      R.push_back((int)C.size());
    }
  return spMtxCRS<T>(m, m, C.size(), R.data(), C.data(), V.data());
}

// irregular rows (some empty, some long), sorted distinct columns
template <class T>
spMtxCRS<T> irregular(int m, int n, unsigned seed) {
  std::mt19937_64 rng(seed);
  std::vector<int> R(1, 0), C;
  std::vector<T> V;
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  for (int r = 0; r < m; ++r) {
    int len = (int)(rng() % 24);
    if (r % 97 == 0) len = 0;
    if (r % 501 == 7) len = 600;
    std::vector<int> cols;
    for (int k = 0; k < len; ++k) cols.push_back((int)(rng() % (uint64_t)n));
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    for (int c : cols) { C.push_back(c); V.push_back((T)u(rng)); }
    R.push_back((int)C.size());
  }
  return spMtxCRS<T>((size_t)m, (size_t)n, C.size(), R.data(), C.data(), V.data());
}

template <class T>
std::vector<double> host_spmv(const spMtxCRS<T>& A, bool trans, double alpha, const std::vector<T>& b, double beta,
                              const std::vector<T>& y0) {
  const size_t rows = trans ? A.n : A.m;
  std::vector<long double> acc(rows, 0.0L);
  for (size_t i = 0; i < A.m; ++i)
    for (int k = A.Rst[i]; k < A.Rst[i + 1]; ++k) {
      if (trans) acc[(size_t)A.Col[k]] += (long double)A.Val[k] * (long double)b[i];
      else acc[i] += (long double)A.Val[k] * (long double)b[(size_t)A.Col[k]];
    }
  std::vector<double> out(rows);
  for (size_t i = 0; i < rows; ++i)
    out[i] = (double)((long double)alpha * acc[i] + (beta == 0.0 ? 0.0L : (long double)beta * (long double)y0[i]));
  return out;
}

template <class T>
double relerr(const std::vector<T>& y, const std::vector<double>& ref) {
  long double num = 0, den = 0;
  for (size_t i = 0; i < ref.size(); ++i) {
    const long double d = (long double)y[i] - (long double)ref[i];
    num += d * d;
    den += (long double)ref[i] * ref[i];
  }
  return den > 0 ? (double)std::sqrt(num / den) : (double)std::sqrt(num);
}

template <class T>
std::vector<T> vec(size_t n, unsigned seed) {
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  std::vector<T> v(n);
  for (auto& e : v) e = (T)u(rng);
  return v;
}

template <class T, template <class> class Mtx>
void product(const char* fmt, const std::string& tag, const spMtxCRS<T>& A, const Mtx<T>& M, double tol) {
  const std::vector<T> b = vec<T>(A.n, 5), y0 = vec<T>(A.m, 6);
  for (double beta : {0.0, -0.5}) {
    std::vector<T> y = y0;
    const sparse_matrix_status st =
        sparse_mv<T, Mtx>(SPARSE_OPERATION_NON_TRANSPOSE, T(1.5), M, sparse_matrix_descr{}, b, T(beta), y);
    const double e = relerr(y, host_spmv(A, false, 1.5, b, beta, y0));
    expect(st.code == 0 && e < tol, std::string(fmt) + " " + tag + " beta=" + std::to_string(beta) +
                                        " code=" + std::to_string(st.code) + " err=" + std::to_string(e));
  }
}

// the mixed-precision extension on a float matrix: error against the exact
// product of the same float values within 1e-6
template <template <class> class Mtx>
void product_mixed(const char* fmt, const std::string& tag, const spMtxCRS<float>& A, const Mtx<float>& M) {
  const std::vector<float> b = vec<float>(A.n, 11), y0 = vec<float>(A.m, 12);
  for (double beta : {0.0, 0.75}) {
    std::vector<float> y = y0;
    const sparse_matrix_status st =
        sparse_mv_mixed<Mtx>(SPARSE_OPERATION_NON_TRANSPOSE, 1.25f, M, sparse_matrix_descr{}, b, (float)beta, y);
    const double e = relerr(y, host_spmv(A, false, 1.25, b, beta, y0));
    expect(st.code == 0 && e < 1e-6, std::string(fmt) + " mixed " + tag + " beta=" + std::to_string(beta) +
                                         " code=" + std::to_string(st.code) + " err=" + std::to_string(e));
  }
}

template <class T>
void run_all(const std::string& tag, const spMtxCRS<T>& A, double tol) {
  product<T, spMtxCRS>("CRS", tag, A, A, tol);
  if constexpr (std::is_same<T, float>::value) product_mixed<spMtxCRS>("CRS", tag, A, A);
  {  // y = A^T b through the transposed CRS
    const std::vector<T> b = vec<T>(A.m, 7), y0 = vec<T>(A.n, 8);
    std::vector<T> y = y0;
    const sparse_matrix_status st =
        sparse_mv<T, spMtxCRS>(SPARSE_OPERATION_TRANSPOSE, T(0.5), A, sparse_matrix_descr{}, b, T(2.0), y);
    const double e = relerr(y, host_spmv(A, true, 0.5, b, 2.0, y0));
    expect(st.code == 0 && e < tol, "CRS transpose " + tag + " err=" + std::to_string(e));
  }
  {
    spMtxHCSR<T> H;
    convertParams p;
    p.param["R"].i = 64;
    p.param["C"].i = 128;
    convert<T, spMtxHCSR>(H, A, p);
    expect(H.values.size() == A.nz && H.block_ptr.back() == (int)A.nz, "HCSR arrays " + tag);
    product<T, spMtxHCSR>("HCSR", tag, A, H, tol);
    if constexpr (std::is_same<T, float>::value) product_mixed<spMtxHCSR>("HCSR", tag, A, H);
  }
  {
    spMtxSELL_C_Sigma<T> S;
    convertParams p;
    p.param["C"].i = 32;
    p.param["Sigma"].i = 128;
    convert<T, spMtxSELL_C_Sigma>(S, A, p);
    product<T, spMtxSELL_C_Sigma>("SELL", tag, A, S, tol);
    if constexpr (std::is_same<T, float>::value) product_mixed<spMtxSELL_C_Sigma>("SELL", tag, A, S);
    // the three stages one after another equal ALL_STAGES
    const std::vector<T> b = vec<T>(A.n, 9), y0 = vec<T>(A.m, 10);
    std::vector<T> y = y0;
    sparse_matrix_status s1 = sparse_mv<T, spMtxSELL_C_Sigma, true, SPARSE_MATRIX_MV_PREPARATION>(
        SPARSE_OPERATION_NON_TRANSPOSE, T(1), S, sparse_matrix_descr{}, b, T(0.25), y);
    sparse_matrix_status s2 = sparse_mv<T, spMtxSELL_C_Sigma, true, SPARSE_MATRIX_MV_MULT>(
        SPARSE_OPERATION_NON_TRANSPOSE, T(1), S, sparse_matrix_descr{}, b, T(0.25), y);
    sparse_matrix_status s3 = sparse_mv<T, spMtxSELL_C_Sigma, true, SPARSE_MATRIX_MV_GET_RESULTS>(
        SPARSE_OPERATION_NON_TRANSPOSE, T(1), S, sparse_matrix_descr{}, b, T(0.25), y);
    const double e = relerr(y, host_spmv(A, false, 1.0, b, 0.25, y0));
    expect(s1.code == 0 && s2.code == 0 && s3.code == 0 && e < tol, "SELL stages " + tag + " err=" + std::to_string(e));
  }
  {
    spMtxCSR5<T> C5;
    convertParams p;
    p.param["sigma"].i = 16;
    convert<T, spMtxCSR5>(C5, A, p);
    expect(C5._omega == 32 && C5._csr_value.size() == A.nz, "CSR5 fields " + tag);
    product<T, spMtxCSR5>("CSR5", tag, A, C5, tol);
    if constexpr (std::is_same<T, float>::value) product_mixed<spMtxCSR5>("CSR5", tag, A, C5);
    spMtxCSR5<T> D;  // the reference's member-function route
    D.inputCSR((int)A.m, (int)A.n, (int)A.nz, A.Rst, A.Col, A.Val);
    expect(D.asCSR5(p) == CSR5_SUCCESS, "CSR5 asCSR5 " + tag);
    product<T, spMtxCSR5>("CSR5(asCSR5)", tag, A, D, tol);
  }
  {
    spMtxLAV<T> L;
    convertParams p;
    p.param["SIMD_Lanes"].i = 8;
    p.param["T"].d = 0.2;
    p.param["segment_len"].i = 300;
    convert<T, spMtxLAV>(L, A, p);
    product<T, spMtxLAV>("LAV", tag, A, L, tol);
  }
  {
    spMtxVNEC<T> V(A);
    product<T, spMtxVNEC>("VNEC", tag, A, V, tol);
  }
  {
    spMtxVHCC<T> W;
    convertParams p;
    p.param["num_threads"].i = 7;
    convert<T, spMtxVHCC>(W, A, p);
    expect(W.get_params().vec_size == 32 && W._thr_info.size() == 7, "VHCC fields " + tag);
    product<T, spMtxVHCC>("VHCC", tag, A, W, tol);
  }
  {
    spMtxCVR<T> R;
    convertParams p;
    p.param["Nthreads"].i = 5;
    convert<T, spMtxCVR>(R, A, p);
    product<T, spMtxCVR>("CVR", tag, A, R, tol);
  }
}

template <class V>
void dump(FILE* f, const std::vector<V>& v) {
  const uint64_t n = v.size();
  std::fwrite(&n, sizeof(n), 1, f);
  if (n) std::fwrite(v.data(), sizeof(V), n, f);
}

}  // namespace

int main(int argc, char** argv) {
  try {
    run_all<double>("laplace64 f64", laplace<double>(64), 1e-12);
    run_all<float>("laplace64 f32", laplace<float>(64), 1e-5);
    run_all<double>("irregular f64", irregular<double>(5000, 4000, 3), 1e-12);
    run_all<float>("irregular f32", irregular<float>(5000, 4000, 4), 1e-5);
    {  // the autotuner's parameters build a format that multiplies correctly
      spMtxCRS<float> A = irregular<float>(20000, 15000, 9);
      const convertParams ph = autotune<float, spMtxHCSR>(A, true, 2);
      spMtxHCSR<float> H;
      convert<float, spMtxHCSR>(H, A, ph);
      product_mixed<spMtxHCSR>("HCSR(tuned)", "irregular f32", A, H);
      const convertParams pc = autotune<float, spMtxCSR5>(A, false, 2);
      spMtxCSR5<float> C5;
      convert<float, spMtxCSR5>(C5, A, pc);
      product<float, spMtxCSR5>("CSR5(tuned)", "irregular f32", A, C5, 1e-5);
      spMtxCRS<double> A64 = irregular<double>(20000, 15000, 10);
      spMtxSELL_C_Sigma<double> S;
      convert<double, spMtxSELL_C_Sigma>(S, A64, autotune<double, spMtxSELL_C_Sigma>(A64, false, 2));
      product<double, spMtxSELL_C_Sigma>("SELL(tuned)", "irregular f64", A64, S, 1e-12);
    }
    {  // reference error behaviour of the HCSR builder
      spMtxHCSR<double> H;
      convertParams p;
      p.param["R"].i = 0;
      bool threw = false;
      try {
        convert<double, spMtxHCSR>(H, laplace<double>(8), p);
      } catch (const std::invalid_argument&) {
        threw = true;
      }
      expect(threw, "HCSR R=0 throws std::invalid_argument");
    }
    if (argc > 1) {  // HCSR with the reference defaults, for comparison with the reference build
      spMtxCRS<double> A = laplace<double>(256);
      spMtxHCSR<double> H;
      convert<double, spMtxHCSR>(H, A, convertParams{});
      FILE* f = std::fopen(argv[1], "wb");
      if (!f) throw std::runtime_error("cannot open output");
      const uint64_t sc[7] = {H.R, H.C, H.m, H.n, H.nz, H.b_m, H.b_n};
      std::fwrite(sc, sizeof(uint64_t), 7, f);
      dump(f, H.block_ptr);
      dump(f, H.row_offset);
      dump(f, H.row_ptr);
      dump(f, H.col_idx);
      dump(f, H.values);
      std::fclose(f);
    }
  } catch (const std::exception& e) {
    std::printf("FAIL exception: %s\n", e.what());
    return 2;
  }
  std::printf("%s (%d failures)\n", failures ? "FAILED" : "OK", failures);
  return failures ? 1 : 0;
}
