// Matrix and eigenpair files.
//
// The reference reads and writes matrices only as CSV text, one matrix row per
// line, element by element through cudaMemcpy (writeMatrixToCsvV2,
// util/inc/fileOpTool.h:51-80; readMatrixFromFile + fillMatrix,
// util/tool/fileOpTool.cu:127-174).  That is too slow for n = 16384 (2 GB of
// doubles), so the library adds a binary record format for clients of the
// solver, and keeps CSV in the reference's layout for small matrices.
//
// Binary file: a sequence of records, each a 32-byte little-endian header
//   char magic[4] = "EVDM"; uint32 version = 1; uint32 elem_bytes = 8;
//   uint32 reserved = 0; int64 rows; int64 cols
// followed by rows * cols FP64 values, column-major.  An eigenpair file holds
// two records: w (n x 1) and X (n x n).
//
// Matrix pointers may be device or host memory (copies use cudaMemcpyDefault);
// columns are staged through a bounded host buffer, several at a time.
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "common.cuh"

namespace evd {
namespace {

struct RecHeader {
  char magic[4];
  uint32_t version;
  uint32_t elem_bytes;
  uint32_t reserved;
  int64_t rows;
  int64_t cols;
};
static_assert(sizeof(RecHeader) == 32, "record header is 32 bytes");

constexpr size_t kStageBytes = size_t(64) << 20;  // host staging per transfer

struct File {
  FILE* f = nullptr;
  File(const char* path, const char* mode) : f(fopen(path, mode)) {}
  ~File() {
    if (f) fclose(f);
  }
};

bool header_ok(const RecHeader& h) {
  return memcmp(h.magic, "EVDM", 4) == 0 && h.version == 1 && h.elem_bytes == 8 && h.rows >= 0 &&
         h.cols >= 0 && (h.rows == 0 || h.cols <= INT64_MAX / 8 / h.rows);
}

bool is_device(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // no device or an unknown pointer: host memory
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// 2-D copy of `height` columns of `width` bytes between host and/or device
// memory; host-to-host copies need no CUDA device.
int copy2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t height) {
  if (!is_device(dst) && !is_device(src)) {
    for (size_t j = 0; j < height; ++j)
      memcpy((char*)dst + j * dpitch, (const char*)src + j * spitch, width);
    return EVD_SUCCESS;
  }
  EVD_CUDA_TRY(cudaMemcpy2D(dst, dpitch, src, spitch, width, height, cudaMemcpyDefault));
  return EVD_SUCCESS;
}

// Columns per staged transfer (at least one).
long cols_per_chunk(long rows) {
  const size_t col = std::max<size_t>(1, (size_t)rows * sizeof(double));
  return (long)std::max<size_t>(1, kStageBytes / col);
}

int write_record(FILE* f, long rows, long cols, const double* A, long ldA) {
  RecHeader h{};
  memcpy(h.magic, "EVDM", 4);
  h.version = 1;
  h.elem_bytes = 8;
  h.rows = rows;
  h.cols = cols;
  if (fwrite(&h, sizeof h, 1, f) != 1) return EVD_ERR_IO;
  if (rows == 0 || cols == 0) return EVD_SUCCESS;
  const long cc = cols_per_chunk(rows);
  std::vector<double> buf((size_t)rows * std::min(cc, cols));
  for (long j0 = 0; j0 < cols; j0 += cc) {
    const long nc = std::min(cc, cols - j0);
    EVD_TRY(copy2d(buf.data(), sizeof(double) * rows, A + (size_t)j0 * ldA,
                   sizeof(double) * ldA, sizeof(double) * rows, nc));
    if (fwrite(buf.data(), sizeof(double) * rows, nc, f) != (size_t)nc) return EVD_ERR_IO;
  }
  return EVD_SUCCESS;
}

// Positions f after the header of record `index`; returns its header.
int seek_record(FILE* f, long index, RecHeader* out) {
  if (index < 0) return EVD_ERR_INVALID_ARG;
  for (long r = 0;; ++r) {
    RecHeader h;
    if (fread(&h, sizeof h, 1, f) != 1) return EVD_ERR_IO;  // past the last record
    if (!header_ok(h)) return EVD_ERR_IO;
    if (r == index) {
      *out = h;
      return EVD_SUCCESS;
    }
    if (fseeko(f, (off_t)(h.rows * h.cols * 8), SEEK_CUR) != 0) return EVD_ERR_IO;
  }
}

int read_record(FILE* f, const RecHeader& h, double* A, long ldA) {
  const long rows = h.rows, cols = h.cols;
  if (rows == 0 || cols == 0) return EVD_SUCCESS;
  const long cc = cols_per_chunk(rows);
  std::vector<double> buf((size_t)rows * std::min(cc, cols));
  for (long j0 = 0; j0 < cols; j0 += cc) {
    const long nc = std::min(cc, cols - j0);
    if (fread(buf.data(), sizeof(double) * rows, nc, f) != (size_t)nc) return EVD_ERR_IO;
    EVD_TRY(copy2d(A + (size_t)j0 * ldA, sizeof(double) * ldA, buf.data(),
                   sizeof(double) * rows, sizeof(double) * rows, nc));
  }
  return EVD_SUCCESS;
}

}  // namespace
}  // namespace evd

using evd::File;
using evd::RecHeader;

static int evd_write_matrix_bin_impl(const char* path, int append, long rows, long cols,
                                    const double* A, long ldA) {
  if (!path || rows < 0 || cols < 0 || (rows * cols > 0 && (!A || ldA < rows)))
    return EVD_ERR_INVALID_ARG;
  File F(path, append ? "ab" : "wb");
  if (!F.f) return EVD_ERR_IO;
  return evd::write_record(F.f, rows, cols, A, ldA);
}

static long evd_matrix_bin_count_impl(const char* path) {
  if (!path) return EVD_ERR_INVALID_ARG;
  File F(path, "rb");
  if (!F.f) return EVD_ERR_IO;
  long count = 0;
  for (;;) {
    RecHeader h;
    const size_t got = fread(&h, 1, sizeof h, F.f);
    if (got == 0 && feof(F.f)) return count;
    if (got != sizeof h || !evd::header_ok(h)) return EVD_ERR_IO;
    if (fseeko(F.f, (off_t)(h.rows * h.cols * 8), SEEK_CUR) != 0) return EVD_ERR_IO;
    ++count;
  }
}

static int evd_matrix_bin_shape_impl(const char* path, long index, long* rows, long* cols) {
  if (!path || !rows || !cols) return EVD_ERR_INVALID_ARG;
  File F(path, "rb");
  if (!F.f) return EVD_ERR_IO;
  RecHeader h;
  EVD_TRY(evd::seek_record(F.f, index, &h));
  *rows = (long)h.rows;
  *cols = (long)h.cols;
  return EVD_SUCCESS;
}

static int evd_read_matrix_bin_impl(const char* path, long index, long rows, long cols, double* A,
                                   long ldA) {
  if (!path || rows < 0 || cols < 0 || (rows * cols > 0 && (!A || ldA < rows)))
    return EVD_ERR_INVALID_ARG;
  File F(path, "rb");
  if (!F.f) return EVD_ERR_IO;
  RecHeader h;
  EVD_TRY(evd::seek_record(F.f, index, &h));
  if (h.rows != rows || h.cols != cols) return EVD_ERR_INVALID_ARG;
  return evd::read_record(F.f, h, A, ldA);
}

static int evd_write_eigenpairs_bin_impl(const char* path, long n, const double* w,
                                        const double* X, long ldX) {
  if (!path || n < 0 || (n > 0 && (!w || !X || ldX < n))) return EVD_ERR_INVALID_ARG;
  File F(path, "wb");
  if (!F.f) return EVD_ERR_IO;
  EVD_TRY(evd::write_record(F.f, n, 1, w, n > 0 ? n : 1));
  return evd::write_record(F.f, n, n, X, ldX);
}

static int evd_read_eigenpairs_bin_impl(const char* path, long n, double* w, double* X, long ldX) {
  if (!path || n < 0 || (n > 0 && (!w || !X || ldX < n))) return EVD_ERR_INVALID_ARG;
  File F(path, "rb");
  if (!F.f) return EVD_ERR_IO;
  RecHeader h;
  EVD_TRY(evd::seek_record(F.f, 0, &h));
  if (h.rows != n || h.cols != 1) return EVD_ERR_INVALID_ARG;
  EVD_TRY(evd::read_record(F.f, h, w, n > 0 ? n : 1));
  if (fread(&h, sizeof h, 1, F.f) != 1 || !evd::header_ok(h)) return EVD_ERR_IO;
  if (h.rows != n || h.cols != n) return EVD_ERR_INVALID_ARG;
  return evd::read_record(F.f, h, X, ldX);
}

// ---- CSV in the reference's layout (one matrix row per line, commas) ----

static int evd_write_matrix_csv_impl(const char* path, long rows, long cols, const double* A,
                                    long ldA) {
  if (!path || rows < 0 || cols < 0 || (rows * cols > 0 && (!A || ldA < rows)))
    return EVD_ERR_INVALID_ARG;
  std::vector<double> h((size_t)rows * cols);
  if (rows * cols > 0)
    EVD_TRY(evd::copy2d(h.data(), sizeof(double) * rows, A, sizeof(double) * ldA,
                   sizeof(double) * rows, cols));
  File F(path, "w");
  if (!F.f) return EVD_ERR_IO;
  for (long i = 0; i < rows; ++i) {
    for (long j = 0; j < cols; ++j)
      if (fprintf(F.f, j + 1 < cols ? "%.17g," : "%.17g", h[i + (size_t)j * rows]) < 0)
        return EVD_ERR_IO;
    if (fputc('\n', F.f) == EOF) return EVD_ERR_IO;
  }
  return EVD_SUCCESS;
}

// Shape query (A == NULL) or read.  Every line must have the same number of
// comma-separated values.
static int evd_read_matrix_csv_impl(const char* path, long* rows, long* cols, double* A, long ldA) {
  if (!path || !rows || !cols) return EVD_ERR_INVALID_ARG;
  File F(path, "r");
  if (!F.f) return EVD_ERR_IO;
  std::vector<double> vals;
  long r = 0, c = -1;
  std::string line;
  for (int ch;;) {
    line.clear();
    while ((ch = fgetc(F.f)) != EOF && ch != '\n') line.push_back((char)ch);
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (!line.empty()) {
      long k = 0;
      const char* p = line.c_str();
      for (;;) {
        char* end;
        const double v = strtod(p, &end);
        if (end == p) return EVD_ERR_IO;
        vals.push_back(v);
        ++k;
        while (*end == ' ' || *end == '\t') ++end;
        if (*end == '\0') break;
        if (*end != ',') return EVD_ERR_IO;
        p = end + 1;
      }
      if (c >= 0 && k != c) return EVD_ERR_IO;
      c = k;
      ++r;
    }
    if (ch == EOF) break;
  }
  if (c < 0) c = 0;
  if (!A) {
    *rows = r;
    *cols = c;
    return EVD_SUCCESS;
  }
  if (*rows != r || *cols != c || ldA < r) return EVD_ERR_INVALID_ARG;
  if (r * c == 0) return EVD_SUCCESS;
  std::vector<double> cm((size_t)r * c);  // row-major text -> column-major
  for (long i = 0; i < r; ++i)
    for (long j = 0; j < c; ++j) cm[i + (size_t)j * r] = vals[(size_t)i * c + j];
  EVD_TRY(evd::copy2d(A, sizeof(double) * ldA, cm.data(), sizeof(double) * r,
                            sizeof(double) * r, c));
  return EVD_SUCCESS;
}

// C ABI wrappers: a C++ exception (host memory for the staging buffers)
// becomes EVD_ERR_HOST.
extern "C" int evd_write_matrix_bin(const char* path, int append, long rows, long cols,
                                    const double* A, long ldA) {
  try {
    return evd_write_matrix_bin_impl(path, append, rows, cols, A, ldA);
  } catch (...) {
    return EVD_ERR_HOST;
  }
}

extern "C" long evd_matrix_bin_count(const char* path) {
  try {
    return evd_matrix_bin_count_impl(path);
  } catch (...) {
    return EVD_ERR_HOST;
  }
}

extern "C" int evd_matrix_bin_shape(const char* path, long index, long* rows, long* cols) {
  try {
    return evd_matrix_bin_shape_impl(path, index, rows, cols);
  } catch (...) {
    return EVD_ERR_HOST;
  }
}

extern "C" int evd_read_matrix_bin(const char* path, long index, long rows, long cols, double* A,
                                   long ldA) {
  try {
    return evd_read_matrix_bin_impl(path, index, rows, cols, A, ldA);
  } catch (...) {
    return EVD_ERR_HOST;
  }
}

extern "C" int evd_write_eigenpairs_bin(const char* path, long n, const double* w,
                                        const double* X, long ldX) {
  try {
    return evd_write_eigenpairs_bin_impl(path, n, w, X, ldX);
  } catch (...) {
    return EVD_ERR_HOST;
  }
}

extern "C" int evd_read_eigenpairs_bin(const char* path, long n, double* w, double* X, long ldX) {
  try {
    return evd_read_eigenpairs_bin_impl(path, n, w, X, ldX);
  } catch (...) {
    return EVD_ERR_HOST;
  }
}

extern "C" int evd_write_matrix_csv(const char* path, long rows, long cols, const double* A,
                                    long ldA) {
  try {
    return evd_write_matrix_csv_impl(path, rows, cols, A, ldA);
  } catch (...) {
    return EVD_ERR_HOST;
  }
}

extern "C" int evd_read_matrix_csv(const char* path, long* rows, long* cols, double* A, long ldA) {
  try {
    return evd_read_matrix_csv_impl(path, rows, cols, A, ldA);
  } catch (...) {
    return EVD_ERR_HOST;
  }
}

