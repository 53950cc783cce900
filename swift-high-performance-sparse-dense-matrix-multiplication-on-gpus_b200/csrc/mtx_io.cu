// mtx_io.cu -- MatrixMarket coordinate files to host CSR (swift_mtx_read in swift_b200.h), the
// reference's on-disk input format.  Host code only.
//
// The CSR is built entry for entry as the reference's reader builds it (mmio_allinone,
// src/auxiliary.h:167-332, over the NIST banner and size parsers of src/mmio.h:142-250):
//   * 1-based indices become 0-based; entries keep FILE order inside each row (no column sort,
//     duplicates kept as separate nonzeros);
//   * "symmetric" and "hermitian" files store one triangle: every off-diagonal entry (i, j)
//     also lands in row j with the same value, placed when the entry is met, so row j sees it
//     in file order among its own entries (src/auxiliary.h:265-300).  "skew-symmetric" is read
//     as stored (the reference mirrors only symmetric and hermitian, :201-205);
//   * pattern entries are 1.0, integer entries their value, complex entries their real part.
// Deviations, each where the reference has no defined result: an index outside [1, M] x [1, N],
// a missing or unparsable entry, an "array" (dense) file and a size line that never comes are
// errors here (the reference reads past them or loops); FP32 values are the double read
// rounded to float (the FP32 reference passes a float to "%lg", test/k-32/FP32/auxiliary.h:65).
#include <cctype>
#include <cerrno>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace swift {
namespace {

struct MtxError {
  swift_status st;
  int ref_code;  // what the reference's mmio_allinone returns at this point
  std::string what;
};

// Whitespace-separated tokens over the file's bytes, as fscanf sees them.
struct Cursor {
  const char *p, *end;
  void skip_ws() {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r' || *p == '\v' || *p == '\f')) ++p;
  }
  bool next_int(long *out) {
    skip_ws();
    if (p >= end) return false;
    char buf[32];
    size_t n = 0;
    while (p + n < end && n < sizeof(buf) - 1 && !isspace((unsigned char)p[n])) ++n;
    memcpy(buf, p, n);
    buf[n] = 0;
    char *e = nullptr;
    errno = 0;
    const long v = strtol(buf, &e, 10);
    if (e == buf || *e != 0 || errno == ERANGE || v < INT_MIN || v > INT_MAX) return false;
    p += n;
    *out = v;
    return true;
  }
  bool next_double(double *out) {
    skip_ws();
    if (p >= end) return false;
    char buf[128];
    size_t n = 0;
    while (p + n < end && n < sizeof(buf) - 1 && !isspace((unsigned char)p[n])) ++n;
    memcpy(buf, p, n);
    buf[n] = 0;
    char *e = nullptr;
    const double v = strtod(buf, &e);
    if (e == buf || *e != 0) return false;
    p += n;
    *out = v;
    return true;
  }
};

enum Field { kReal, kComplex, kPattern, kInteger };

struct Parsed {
  int M = 0, N = 0, nz = 0;
  bool symmetric = false;
  std::vector<int> row, col;
  std::vector<double> val;
};

std::string lower(std::string s) {
  for (char &c : s) c = (char)tolower((unsigned char)c);
  return s;
}

// Banner (src/mmio.h:172-250), size line (:142-170), then nz entries.
void parse(const char *data, size_t size, Parsed &out) {
  const char *p = data, *end = data + size;
  const char *eol = (const char *)memchr(p, '\n', size);
  std::string line(p, eol ? eol : end);
  char tok[5][64];
  if (sscanf(line.c_str(), "%63s %63s %63s %63s %63s", tok[0], tok[1], tok[2], tok[3], tok[4]) != 5)
    throw MtxError{SWIFT_ERR_FORMAT, -2, "the first line is not a MatrixMarket banner"};
  if (strncmp(tok[0], "%%MatrixMarket", 14) != 0)
    throw MtxError{SWIFT_ERR_FORMAT, -2, "missing %%MatrixMarket banner"};
  const std::string obj = lower(tok[1]), fmt = lower(tok[2]), field = lower(tok[3]), sym = lower(tok[4]);
  if (obj != "matrix") throw MtxError{SWIFT_ERR_FORMAT, -2, "object is not 'matrix'"};
  if (fmt == "array")
    throw MtxError{SWIFT_ERR_UNSUPPORTED, -2, "'array' (dense) MatrixMarket files are not sparse inputs"};
  if (fmt != "coordinate") throw MtxError{SWIFT_ERR_FORMAT, -2, "format is neither 'coordinate' nor 'array'"};
  Field f;
  if (field == "real") f = kReal;
  else if (field == "complex") f = kComplex;
  else if (field == "pattern") f = kPattern;
  else if (field == "integer") f = kInteger;
  else throw MtxError{SWIFT_ERR_FORMAT, -2, "unknown field type"};
  if (sym == "symmetric" || sym == "hermitian") out.symmetric = true;
  else if (sym != "general" && sym != "skew-symmetric") throw MtxError{SWIFT_ERR_FORMAT, -2, "unknown symmetry"};

  // comment lines start with '%'; the size line is the first other line (a blank one makes
  // the reference scan on for three integers, as the cursor does)
  p = eol ? eol + 1 : end;
  while (p < end && *p == '%') {
    const char *e = (const char *)memchr(p, '\n', (size_t)(end - p));
    p = e ? e + 1 : end;
  }
  Cursor c{p, end};
  long M, N, nz;
  if (!c.next_int(&M) || !c.next_int(&N) || !c.next_int(&nz))
    throw MtxError{SWIFT_ERR_FORMAT, -4, "missing or malformed size line"};
  if (M < 0 || N < 0 || nz < 0) throw MtxError{SWIFT_ERR_FORMAT, -4, "negative size"};
  out.M = (int)M;
  out.N = (int)N;
  out.nz = (int)nz;
  out.row.resize(nz);
  out.col.resize(nz);
  out.val.resize(nz);
  for (long i = 0; i < nz; ++i) {
    long r, k;
    double v = 1.0, im;
    bool ok = c.next_int(&r) && c.next_int(&k);
    if (ok) {
      switch (f) {
        case kReal: ok = c.next_double(&v); break;
        case kComplex: ok = c.next_double(&v) && c.next_double(&im); break;
        case kInteger: {
          long iv;
          ok = c.next_int(&iv);
          v = (double)iv;
          break;
        }
        case kPattern: break;
      }
    }
    if (!ok) throw MtxError{SWIFT_ERR_FORMAT, -5, "entry " + std::to_string(i + 1) + " is missing or malformed"};
    if (r < 1 || r > M || k < 1 || k > N)
      throw MtxError{SWIFT_ERR_FORMAT, -5, "entry " + std::to_string(i + 1) + " has an index outside the matrix"};
    out.row[i] = (int)(r - 1);
    out.col[i] = (int)(k - 1);
    out.val[i] = v;
  }
}

template <class T>
swift_status build_csr(const Parsed &in, int **rowptr, int **colidx, T **val, int *nnz_out) {
  const int M = in.M;
  const size_t nz = in.row.size();
  std::vector<int64_t> cnt((size_t)M + 1, 0);
  for (size_t i = 0; i < nz; ++i) {
    cnt[in.row[i]]++;
    // a mirrored entry needs a row of the same index: square matrices, as symmetry implies
    if (in.symmetric && in.row[i] != in.col[i]) {
      if (in.col[i] >= M) {
        set_last_error("swift_mtx_read", "symmetric file with an entry outside the square part");
        return SWIFT_ERR_FORMAT;
      }
      cnt[in.col[i]]++;
    }
  }
  int64_t run = 0;
  for (int r = 0; r <= M; ++r) {
    const int64_t c = cnt[r];
    cnt[r] = run;
    run += c;
  }
  if (run > INT_MAX) {
    set_last_error("swift_mtx_read", "expanded nonzero count exceeds the int32 range");
    return SWIFT_ERR_OVERFLOW;
  }
  int *rp = static_cast<int *>(malloc(sizeof(int) * ((size_t)M + 1)));
  int *ci = static_cast<int *>(malloc(sizeof(int) * (run ? (size_t)run : 1)));
  T *vv = static_cast<T *>(malloc(sizeof(T) * (run ? (size_t)run : 1)));
  if (!rp || !ci || !vv) {
    free(rp);
    free(ci);
    free(vv);
    set_last_error("swift_mtx_read", "host allocation failed");
    return SWIFT_ERR_ALLOC;
  }
  for (int r = 0; r <= M; ++r) rp[r] = (int)cnt[r];
  std::vector<int> fill((size_t)M, 0);
  auto put = [&](int r, int c, double v) {
    const int64_t o = rp[r] + fill[r]++;
    ci[o] = c;
    vv[o] = (T)v;
  };
  for (size_t i = 0; i < nz; ++i) {
    put(in.row[i], in.col[i], in.val[i]);
    if (in.symmetric && in.row[i] != in.col[i]) put(in.col[i], in.row[i], in.val[i]);
  }
  *rowptr = rp;
  *colidx = ci;
  *val = vv;
  *nnz_out = (int)run;
  return SWIFT_OK;
}

}  // namespace
}  // namespace swift

using namespace swift;

extern "C" {

swift_status swift_mtx_read(const char *path, swift_dtype val_type, int *m, int *n, int *nnz,
                            int *is_symmetric, int **rowptr, int **colidx, void **val, int *reference_code) {
  if (reference_code) *reference_code = 0;
  if (!path || !m || !n || !nnz || !is_symmetric || !rowptr || !colidx || !val ||
      (val_type != SWIFT_F32 && val_type != SWIFT_F64)) {
    set_last_error("swift_mtx_read", "null argument or value type other than F32/F64");
    return SWIFT_ERR_INVALID_ARG;
  }
  *rowptr = nullptr;
  *colidx = nullptr;
  *val = nullptr;
  FILE *f = fopen(path, "rb");
  if (!f) {
    if (reference_code) *reference_code = -1;
    set_last_error("swift_mtx_read", (std::string("cannot open ") + path).c_str());
    return SWIFT_ERR_IO;
  }
  std::vector<char> data;
  char buf[1 << 16];
  size_t got;
  while ((got = fread(buf, 1, sizeof(buf), f)) > 0) data.insert(data.end(), buf, buf + got);
  const bool read_err = ferror(f) != 0;
  fclose(f);
  if (read_err) {
    if (reference_code) *reference_code = -1;
    set_last_error("swift_mtx_read", "read error");
    return SWIFT_ERR_IO;
  }
  Parsed in;
  try {
    parse(data.data(), data.size(), in);
  } catch (const MtxError &e) {
    if (reference_code) *reference_code = e.ref_code;
    set_last_error("swift_mtx_read", e.what.c_str());
    return e.st;
  } catch (const std::bad_alloc &) {
    set_last_error("swift_mtx_read", "host allocation failed");
    return SWIFT_ERR_ALLOC;
  }
  swift_status st = val_type == SWIFT_F64
                        ? build_csr<double>(in, rowptr, colidx, reinterpret_cast<double **>(val), nnz)
                        : build_csr<float>(in, rowptr, colidx, reinterpret_cast<float **>(val), nnz);
  if (st != SWIFT_OK) {
    if (reference_code) *reference_code = -5;
    return st;
  }
  *m = in.M;
  *n = in.N;
  *is_symmetric = in.symmetric ? 1 : 0;
  return SWIFT_OK;
}

void swift_host_free(void *p) { free(p); }

}  // extern "C"
