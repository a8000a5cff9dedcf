// mmio.cpp — on-disk sparse matrices on the host: the Matrix Market
// coordinate format (the reference's spMtxCRS carries an MM_typecode,
// include/CRS.h:8,17, but ships no reader) and a binary CRS container, the
// "mtx to bin" conversion its test environment names
// (cmake/TestEnvironment.cmake:62).
//
// Reader: the whole file is read into memory and parsed with strtoll/strtod;
// "real", "integer" and "pattern" fields (pattern entries get the value 1),
// "general", "symmetric" and "skew-symmetric" symmetry (the mirror entry of
// an off-diagonal (i, j, v) is (j, i, v) or (j, i, -v)).  Entries become CRS
// with every row's columns ascending; duplicates of one (row, column) are
// summed in file order.  Complex, Hermitian and dense "array" files are
// rejected (RVVLA_ERR_UNSUPPORTED).
//
// Binary CRS: a 48-byte little-endian header — "RVVLACRS", u32 version 1,
// u32 value bytes (8 or 4), i64 m, i64 n, i64 nz, i64 reserved 0 — then
// Rst int32[m+1], Col int32[nz], Val[nz].  The reader checks the magic, the
// version, the sizes against the file length and the row pointers.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "rvvla.h"

namespace rvvla {
int fail(int status, const std::string& msg);
}

namespace {

using rvvla::fail;

bool read_file(const char* path, std::string& out) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  out.clear();
  char buf[1 << 16];
  size_t k;
  while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) out.append(buf, k);
  const bool ok = !std::ferror(f);
  std::fclose(f);
  return ok;
}

std::string lower(std::string s) {
  for (char& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

// next line [p, eol) of the buffer; advances p past the newline
bool next_line(const char*& p, const char* end, const char*& b, const char*& e) {
  if (p >= end) return false;
  b = p;
  const void* nl = std::memchr(p, '\n', (size_t)(end - p));
  e = nl ? static_cast<const char*>(nl) : end;
  p = nl ? e + 1 : end;
  return true;
}

bool blank(const char* b, const char* e) {
  for (; b < e; ++b)
    if (!std::isspace((unsigned char)*b)) return false;
  return true;
}

struct Triple {
  int32_t r, c;
  double v;
};

int to_crs(int64_t m, std::vector<Triple>& t, rvvla_host_crs* out) {
  std::vector<int64_t> cnt((size_t)m + 1, 0);
  for (const Triple& x : t) cnt[(size_t)x.r + 1]++;
  for (int64_t i = 0; i < m; ++i) cnt[(size_t)i + 1] += cnt[(size_t)i];
  std::vector<Triple> byrow(t.size());
  {
    std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
    for (const Triple& x : t) byrow[(size_t)pos[(size_t)x.r]++] = x;  // file order inside a row
  }
  t.clear();
  t.shrink_to_fit();
  // sort each row by column (stable: duplicates keep file order), merge duplicates
  std::vector<int32_t> rst((size_t)m + 1, 0);
  std::vector<int32_t> col;
  std::vector<double> val;
  col.reserve(byrow.size());
  val.reserve(byrow.size());
  for (int64_t i = 0; i < m; ++i) {
    auto b = byrow.begin() + cnt[(size_t)i], e = byrow.begin() + cnt[(size_t)i + 1];
    std::stable_sort(b, e, [](const Triple& a, const Triple& c) { return a.c < c.c; });
    for (auto it = b; it != e; ++it) {
      if (!col.empty() && (int64_t)col.size() > rst[(size_t)i] && col.back() == it->c) val.back() += it->v;
      else {
        col.push_back(it->c);
        val.push_back(it->v);
      }
    }
    rst[(size_t)i + 1] = (int32_t)col.size();
  }
  out->nz = (int64_t)col.size();
  out->Rst = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (size_t)(m + 1)));
  out->Col = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * std::max<size_t>(col.size(), 1)));
  out->Val = static_cast<double*>(std::malloc(sizeof(double) * std::max<size_t>(val.size(), 1)));
  if (!out->Rst || !out->Col || !out->Val) {
    rvvla_host_crs_free(out);
    return fail(RVVLA_ERR_TOO_LARGE, "matrix market: out of host memory");
  }
  std::memcpy(out->Rst, rst.data(), sizeof(int32_t) * rst.size());
  if (!col.empty()) {
    std::memcpy(out->Col, col.data(), sizeof(int32_t) * col.size());
    std::memcpy(out->Val, val.data(), sizeof(double) * val.size());
  }
  return RVVLA_OK;
}

struct BinHeader {
  char magic[8];
  uint32_t version, val_bytes;
  int64_t m, n, nz, reserved;
};
static_assert(sizeof(BinHeader) == 48, "binary CRS header is 48 bytes");

}  // namespace

extern "C" {

void rvvla_host_crs_free(rvvla_host_crs* A) {
  if (!A) return;
  std::free(A->Rst);
  std::free(A->Col);
  std::free(A->Val);
  A->Rst = nullptr;
  A->Col = nullptr;
  A->Val = nullptr;
}

int rvvla_mm_read(const char* path, rvvla_host_crs* out) {
  if (!path || !out) return fail(RVVLA_ERR_INVALID_ARG, "mm_read: null argument");
  std::memset(out, 0, sizeof(*out));
  std::string buf;
  if (!read_file(path, buf)) return fail(RVVLA_ERR_IO, std::string("mm_read: cannot read ") + path);
  const char* p = buf.data();
  const char* end = p + buf.size();
  const char *b, *e;
  if (!next_line(p, end, b, e)) return fail(RVVLA_ERR_FORMAT, "matrix market: empty file");
  // banner: %%MatrixMarket matrix coordinate <field> <symmetry>
  char w[5][64] = {};
  {
    std::string head(b, e);
    if (std::sscanf(head.c_str(), "%63s %63s %63s %63s %63s", w[0], w[1], w[2], w[3], w[4]) != 5 ||
        lower(w[0]) != "%%matrixmarket" || lower(w[1]) != "matrix")
      return fail(RVVLA_ERR_FORMAT, "matrix market: missing '%%MatrixMarket matrix ...' banner");
  }
  const std::string fmt = lower(w[2]), field = lower(w[3]), sym = lower(w[4]);
  if (fmt != "coordinate") return fail(RVVLA_ERR_UNSUPPORTED, "matrix market: only the coordinate format is read");
  int fld;
  if (field == "real" || field == "double") fld = 0;
  else if (field == "integer") fld = 1;
  else if (field == "pattern") fld = 2;
  else return fail(RVVLA_ERR_UNSUPPORTED, "matrix market: field '" + field + "' is not real, integer or pattern");
  int sy;
  if (sym == "general") sy = 0;
  else if (sym == "symmetric") sy = 1;
  else if (sym == "skew-symmetric") sy = 2;
  else return fail(RVVLA_ERR_UNSUPPORTED, "matrix market: symmetry '" + sym + "' is not supported");
  // size line (after comments)
  long long M = -1, N = -1, L = -1;
  while (next_line(p, end, b, e)) {
    if (b < e && *b == '%') continue;
    if (blank(b, e)) continue;
    std::string sz(b, e);
    if (std::sscanf(sz.c_str(), "%lld %lld %lld", &M, &N, &L) != 3 || M < 0 || N < 0 || L < 0)
      return fail(RVVLA_ERR_FORMAT, "matrix market: bad size line");
    break;
  }
  if (M < 0) return fail(RVVLA_ERR_FORMAT, "matrix market: no size line");
  if (M >= INT32_MAX || N >= INT32_MAX) return fail(RVVLA_ERR_TOO_LARGE, "matrix market: dimensions beyond int32");
  if ((sy != 0) && M != N) return fail(RVVLA_ERR_FORMAT, "matrix market: a symmetric matrix must be square");
  std::vector<Triple> t;
  t.reserve((size_t)(sy ? 2 * L : L));
  long long got = 0;
  while (got < L && next_line(p, end, b, e)) {
    if (blank(b, e) || *b == '%') continue;
    std::string ln(b, e);
    const char* s = ln.c_str();
    char* q;
    errno = 0;
    const long long i = std::strtoll(s, &q, 10);
    if (q == s) return fail(RVVLA_ERR_FORMAT, "matrix market: bad entry line " + std::to_string(got + 1));
    s = q;
    const long long j = std::strtoll(s, &q, 10);
    if (q == s) return fail(RVVLA_ERR_FORMAT, "matrix market: bad entry line " + std::to_string(got + 1));
    s = q;
    double v = 1.0;
    if (fld != 2) {
      v = std::strtod(s, &q);
      if (q == s) return fail(RVVLA_ERR_FORMAT, "matrix market: missing value on entry " + std::to_string(got + 1));
    }
    if (i < 1 || i > M || j < 1 || j > N)
      return fail(RVVLA_ERR_FORMAT, "matrix market: entry " + std::to_string(got + 1) + " outside the matrix");
    t.push_back({(int32_t)(i - 1), (int32_t)(j - 1), v});
    if (sy && i != j) t.push_back({(int32_t)(j - 1), (int32_t)(i - 1), sy == 2 ? -v : v});
    if (sy == 2 && i == j && v != 0.0)
      return fail(RVVLA_ERR_FORMAT, "matrix market: a skew-symmetric matrix has a nonzero diagonal entry");
    ++got;
  }
  if (got != L)
    return fail(RVVLA_ERR_FORMAT, "matrix market: " + std::to_string(L) + " entries announced, " +
                                      std::to_string(got) + " found");
  if ((long long)t.size() >= INT32_MAX) return fail(RVVLA_ERR_TOO_LARGE, "matrix market: more nonzeros than int32");
  out->m = M;
  out->n = N;
  return to_crs(M, t, out);
}

int rvvla_mm_write(const char* path, int64_t m, int64_t n, const int32_t* Rst, const int32_t* Col,
                   const double* Val) {
  if (!path || m < 0 || n < 0 || !Rst || (Rst[m] > 0 && (!Col || !Val)))
    return fail(RVVLA_ERR_INVALID_ARG, "mm_write: bad argument");
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(RVVLA_ERR_IO, std::string("mm_write: cannot open ") + path);
  bool ok = std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%lld %lld %lld\n", (long long)m,
                         (long long)n, (long long)Rst[m]) > 0;
  char line[96];
  for (int64_t i = 0; ok && i < m; ++i)
    for (int32_t k = Rst[i]; ok && k < Rst[i + 1]; ++k) {
      const int len = std::snprintf(line, sizeof(line), "%lld %d %.17g\n", (long long)(i + 1), Col[k] + 1, Val[k]);
      ok = std::fwrite(line, 1, (size_t)len, f) == (size_t)len;
    }
  ok = (std::fclose(f) == 0) && ok;
  return ok ? RVVLA_OK : fail(RVVLA_ERR_IO, std::string("mm_write: write failed on ") + path);
}

int rvvla_crs_save(const char* path, int64_t m, int64_t n, int64_t nz, const int32_t* Rst, const int32_t* Col,
                   const void* Val, int val_bytes) {
  if (!path || m < 0 || n < 0 || nz < 0 || !Rst || (nz > 0 && (!Col || !Val)) || (val_bytes != 8 && val_bytes != 4))
    return fail(RVVLA_ERR_INVALID_ARG, "crs_save: bad argument");
  if (Rst[0] != 0 || Rst[m] != nz) return fail(RVVLA_ERR_FORMAT, "crs_save: Rst[0] must be 0 and Rst[m] = nz");
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(RVVLA_ERR_IO, std::string("crs_save: cannot open ") + path);
  BinHeader h{};
  std::memcpy(h.magic, "RVVLACRS", 8);
  h.version = 1;
  h.val_bytes = (uint32_t)val_bytes;
  h.m = m;
  h.n = n;
  h.nz = nz;
  bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 &&
            std::fwrite(Rst, sizeof(int32_t), (size_t)m + 1, f) == (size_t)m + 1 &&
            (nz == 0 || (std::fwrite(Col, sizeof(int32_t), (size_t)nz, f) == (size_t)nz &&
                         std::fwrite(Val, (size_t)val_bytes, (size_t)nz, f) == (size_t)nz));
  ok = (std::fclose(f) == 0) && ok;
  return ok ? RVVLA_OK : fail(RVVLA_ERR_IO, std::string("crs_save: write failed on ") + path);
}

int rvvla_crs_load_info(const char* path, int64_t* m, int64_t* n, int64_t* nz, int* val_bytes) {
  if (!path || !m || !n || !nz || !val_bytes) return fail(RVVLA_ERR_INVALID_ARG, "crs_load_info: null argument");
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(RVVLA_ERR_IO, std::string("crs_load: cannot open ") + path);
  BinHeader h{};
  const bool got = std::fread(&h, sizeof(h), 1, f) == 1;
  std::fseek(f, 0, SEEK_END);
  const long long size = std::ftell(f);
  std::fclose(f);
  if (!got || std::memcmp(h.magic, "RVVLACRS", 8) != 0) return fail(RVVLA_ERR_FORMAT, "crs_load: not a binary CRS file");
  if (h.version != 1) return fail(RVVLA_ERR_UNSUPPORTED, "crs_load: unknown version " + std::to_string(h.version));
  if ((h.val_bytes != 8 && h.val_bytes != 4) || h.m < 0 || h.n < 0 || h.nz < 0 || h.m >= INT32_MAX ||
      h.nz >= INT32_MAX)
    return fail(RVVLA_ERR_FORMAT, "crs_load: bad header");
  const long long want = (long long)sizeof(h) + 4LL * (h.m + 1) + (4LL + h.val_bytes) * h.nz;
  if (size != want) return fail(RVVLA_ERR_FORMAT, "crs_load: file length does not match its header");
  *m = h.m;
  *n = h.n;
  *nz = h.nz;
  *val_bytes = (int)h.val_bytes;
  return RVVLA_OK;
}

int rvvla_crs_load(const char* path, int32_t* Rst, int32_t* Col, void* Val) {
  int64_t m, n, nz;
  int vb;
  int rc = rvvla_crs_load_info(path, &m, &n, &nz, &vb);
  if (rc) return rc;
  if (!Rst || (nz > 0 && (!Col || !Val))) return fail(RVVLA_ERR_INVALID_ARG, "crs_load: null array");
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(RVVLA_ERR_IO, std::string("crs_load: cannot open ") + path);
  bool ok = std::fseek(f, (long)sizeof(BinHeader), SEEK_SET) == 0 &&
            std::fread(Rst, sizeof(int32_t), (size_t)m + 1, f) == (size_t)m + 1 &&
            (nz == 0 || (std::fread(Col, sizeof(int32_t), (size_t)nz, f) == (size_t)nz &&
                         std::fread(Val, (size_t)vb, (size_t)nz, f) == (size_t)nz));
  std::fclose(f);
  if (!ok) return fail(RVVLA_ERR_IO, std::string("crs_load: read failed on ") + path);
  if (Rst[0] != 0 || Rst[m] != nz) return fail(RVVLA_ERR_FORMAT, "crs_load: row pointers do not span the nonzeros");
  for (int64_t i = 0; i < m; ++i)
    if (Rst[i + 1] < Rst[i]) return fail(RVVLA_ERR_FORMAT, "crs_load: row pointers decrease");
  for (int64_t k = 0; k < nz; ++k)
    if (Col[k] < 0 || Col[k] >= n) return fail(RVVLA_ERR_FORMAT, "crs_load: column index outside the matrix");
  return RVVLA_OK;
}

}  // extern "C"
