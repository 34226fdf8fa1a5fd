// Files in the reference's formats (host code only).
//
//   vector files   RealVector::WriteVector / ReadVector (src/Vector/RealVector.cc:3669, :3798):
//                  little-endian int32 dimension, or int32 -1 and an int64 dimension from 2^31 on,
//                  then the components as little-endian doubles.
//   lanczos.dat    the state files of BasicLanczosAlgorithmWithDiskStorage
//                  (src/LanczosAlgorithm/BasicLanczosAlgorithmWithDiskStorage.cc:286-335) and of
//                  BasicLanczosAlgorithmWithGroundStateDiskStorage (...WithGroundStateDiskStorage.cc:
//                  399-453), field by field in the same order and widths.
//
// Every file is written to "<name>.tmp" and renamed into place, so a reader never sees a torn file.
#include <errno.h>
#include <stdio.h>
#include <string.h>
#include <unistd.h>

#include <algorithm>
#include <string>
#include <vector>

#include "dh_disk.h"
#include "dh_internal.h"
#include "dh_objects.h"

#if !defined(__BYTE_ORDER__) || __BYTE_ORDER__ != __ORDER_LITTLE_ENDIAN__
#error "the reference's files are little-endian: this code writes native doubles and integers"
#endif

namespace dh {

namespace {

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

int io_fail(const std::string& path, const char* what) {
  set_error("%s %s: %s", what, path.c_str(), errno ? strerror(errno) : "unexpected end of file");
  return DH_ERR_IO;
}

bool put(FILE* f, const void* p, size_t n) { return n == 0 || fwrite(p, 1, n, f) == n; }
bool get(FILE* f, void* p, size_t n) { return n == 0 || fread(p, 1, n, f) == n; }

// size of an open file (seek to the end and back)
long long file_size(FILE* f) {
  if (fseeko(f, 0, SEEK_END) != 0) return -1;
  const long long n = (long long)ftello(f);
  if (fseeko(f, 0, SEEK_SET) != 0) return -1;
  return n;
}

int finish_write(File& out, const std::string& tmp, const std::string& path) {
  errno = 0;
  const bool ok = fflush(out.f) == 0 && fsync(fileno(out.f)) == 0;
  const int closed = fclose(out.f);
  out.f = nullptr;
  if (!ok || closed != 0) {
    remove(tmp.c_str());
    return io_fail(tmp, "cannot write");
  }
  if (rename(tmp.c_str(), path.c_str()) != 0) {
    remove(tmp.c_str());
    return io_fail(path, "cannot rename into");
  }
  return DH_OK;
}

}  // namespace

std::string join_path(const std::string& directory, const char* name) {
  if (directory.empty()) return name;
  if (directory.back() == '/') return directory + name;
  return directory + "/" + name;
}

int vector_file_write(const std::string& path, const double* v, int64_t dim, int per) {
  DH_CHECK(dim >= 0, DH_ERR_ARGUMENT, "negative vector dimension");
  const std::string tmp = path + ".tmp";
  File out;
  errno = 0;
  out.f = fopen(tmp.c_str(), "wb");
  if (!out.f) return io_fail(tmp, "cannot open");
  bool ok;
  if (dim < (int64_t(1) << 31)) {
    const int32_t d = (int32_t)dim;
    ok = put(out.f, &d, 4);
  } else {
    const int32_t flag = -1;
    ok = put(out.f, &flag, 4) && put(out.f, &dim, 8);
  }
  ok = ok && put(out.f, v, (size_t)dim * per * sizeof(double));
  if (!ok) {
    fclose(out.f);
    out.f = nullptr;
    remove(tmp.c_str());
    return io_fail(tmp, "cannot write");
  }
  return finish_write(out, tmp, path);
}

// header of a vector file: dimension and offset of the first component; checks the file length
static int vector_file_header(FILE* f, const std::string& path, int64_t* dim, long long* offset, int per) {
  const long long size = file_size(f);
  if (size < 4) return io_fail(path, "not a vector file (too short):");
  int32_t d32 = 0;
  if (!get(f, &d32, 4)) return io_fail(path, "cannot read");
  int64_t d = d32;
  long long off = 4;
  if (d32 <= 0) {
    // RealVector::ReadVector reads the int64 dimension whenever the int32 one is not positive; an
    // empty vector is written with a bare 0
    if (d32 == 0 && size == 4) {
      *dim = 0;
      *offset = 4;
      return DH_OK;
    }
    if (!get(f, &d, 8)) return io_fail(path, "cannot read");
    off = 12;
    DH_CHECK(d >= 0, DH_ERR_IO, "%s: negative vector dimension %lld", path.c_str(), (long long)d);
  }
  DH_CHECK(size == off + d * per * (long long)sizeof(double), DH_ERR_IO,
           "%s: %lld bytes do not hold a %s vector of dimension %lld", path.c_str(), size,
           per == 2 ? "complex" : "real", (long long)d);
  *dim = d;
  *offset = off;
  return DH_OK;
}

int vector_file_dimension(const std::string& path, int64_t* dim, int per) {
  File in;
  errno = 0;
  in.f = fopen(path.c_str(), "rb");
  if (!in.f) return io_fail(path, "cannot open");
  long long off = 0;
  return vector_file_header(in.f, path, dim, &off, per);
}

int vector_file_read(const std::string& path, double* v, int64_t dim, int per) {
  File in;
  errno = 0;
  in.f = fopen(path.c_str(), "rb");
  if (!in.f) return io_fail(path, "cannot open");
  int64_t d = 0;
  long long off = 0;
  int rc = vector_file_header(in.f, path, &d, &off, per);
  if (rc != DH_OK) return rc;
  DH_CHECK(d == dim, DH_ERR_IO, "%s holds a vector of dimension %lld, expected %lld", path.c_str(), (long long)d,
           (long long)dim);
  if (fseeko(in.f, off, SEEK_SET) != 0 || !get(in.f, v, (size_t)dim * per * sizeof(double)))
    return io_fail(path, "cannot read");
  return DH_OK;
}

int lanczos_state_write(const std::string& path, int algorithm, const LanczosDiskState& s) {
  const int rows = (int)s.diag.size();
  DH_CHECK((int)s.upper.size() + 1 == rows || (rows == 0 && s.upper.empty()), DH_ERR_ARGUMENT,
           "tridiagonal matrix with %d diagonal and %d upper-diagonal elements", rows, (int)s.upper.size());
  const std::string tmp = path + ".tmp";
  File out;
  errno = 0;
  out.f = fopen(tmp.c_str(), "wb");
  if (!out.f) return io_fail(tmp, "cannot open");
  bool ok = true;
  if (algorithm == DH_LANCZOS_BASIC) {
    // Index, PreviousLastWantedEigenvalue, EigenvaluePrecision, NbrRow, three NUL-terminated vector
    // file names, diagonal 0..Index+1, upper diagonal 0..Index
    DH_CHECK(rows == s.index + 2, DH_ERR_ARGUMENT, "basic state: %d rows for Index %d", rows, s.index);
    ok = put(out.f, &s.index, 4) && put(out.f, &s.prev_last, 8) && put(out.f, &s.precision, 8) &&
         put(out.f, &s.nbr_row, 4);
    for (int k = 0; k < 3 && ok; ++k) ok = put(out.f, s.names[k], strlen(s.names[k]) + 1);
    ok = ok && put(out.f, s.diag.data(), (size_t)(s.index + 2) * 8) && put(out.f, s.upper.data(), (size_t)(s.index + 1) * 8);
  } else {
    // Index, GroundStateEvaluationFlag, PreviousLastWantedEigenvalue, EigenvaluePrecision,
    // NbrEigenvalue, NbrRow, diagonal 0..NbrRow-1, upper diagonal 0..NbrRow-2
    DH_CHECK(rows == s.nbr_row, DH_ERR_ARGUMENT, "ground-state format: %d rows stored as %d", rows, s.nbr_row);
    ok = put(out.f, &s.index, 4) && put(out.f, &s.ground_flag, 4) && put(out.f, &s.prev_last, 8) &&
         put(out.f, &s.precision, 8) && put(out.f, &s.nbr_eigenvalue, 4) && put(out.f, &s.nbr_row, 4) &&
         put(out.f, s.diag.data(), (size_t)rows * 8) && put(out.f, s.upper.data(), (size_t)std::max(rows - 1, 0) * 8);
  }
  if (!ok) {
    fclose(out.f);
    out.f = nullptr;
    remove(tmp.c_str());
    return io_fail(tmp, "cannot write");
  }
  return finish_write(out, tmp, path);
}

int lanczos_state_read(const std::string& path, int algorithm, LanczosDiskState* s) {
  File in;
  errno = 0;
  in.f = fopen(path.c_str(), "rb");
  if (!in.f) return io_fail(path, "cannot open");
  const long long size = file_size(in.f);
  long long expect = 0;
  if (algorithm == DH_LANCZOS_BASIC) {
    if (!get(in.f, &s->index, 4) || !get(in.f, &s->prev_last, 8) || !get(in.f, &s->precision, 8) ||
        !get(in.f, &s->nbr_row, 4))
      return io_fail(path, "cannot read");
    // the reader of the reference takes 8 bytes per name ("vectorN" and its NUL)
    for (int k = 0; k < 3; ++k) {
      if (!get(in.f, s->names[k], 8)) return io_fail(path, "cannot read");
      DH_CHECK(memchr(s->names[k], 0, 8) != nullptr && s->names[k][0] != 0 && strchr(s->names[k], '/') == nullptr,
               DH_ERR_IO, "%s: bad vector file name", path.c_str());
    }
    DH_CHECK(s->index >= 0 && s->index < (1 << 28) && s->nbr_row >= s->index + 2, DH_ERR_IO,
             "%s: Index %d with %d rows", path.c_str(), s->index, s->nbr_row);
    const int rows = s->index + 2;
    s->diag.resize(rows);
    s->upper.resize(rows - 1);
    if (!get(in.f, s->diag.data(), (size_t)rows * 8) || !get(in.f, s->upper.data(), (size_t)(rows - 1) * 8))
      return io_fail(path, "cannot read");
    s->ground_flag = 0;
    s->nbr_eigenvalue = 0;
    expect = 24 + 24 + 8LL * rows + 8LL * (rows - 1);
  } else {
    if (!get(in.f, &s->index, 4) || !get(in.f, &s->ground_flag, 4) || !get(in.f, &s->prev_last, 8) ||
        !get(in.f, &s->precision, 8) || !get(in.f, &s->nbr_eigenvalue, 4) || !get(in.f, &s->nbr_row, 4))
      return io_fail(path, "cannot read");
    DH_CHECK(s->nbr_row >= 2 && s->nbr_row < (1 << 28) && s->index >= 0 && (s->ground_flag == 0 || s->ground_flag == 1),
             DH_ERR_IO, "%s: Index %d, flag %d, %d rows", path.c_str(), s->index, s->ground_flag, s->nbr_row);
    DH_CHECK(s->ground_flag == 1 || s->nbr_row >= s->index + 2, DH_ERR_IO, "%s: Index %d with %d rows", path.c_str(),
             s->index, s->nbr_row);
    s->diag.resize(s->nbr_row);
    s->upper.resize(s->nbr_row - 1);
    if (!get(in.f, s->diag.data(), (size_t)s->nbr_row * 8) || !get(in.f, s->upper.data(), (size_t)(s->nbr_row - 1) * 8))
      return io_fail(path, "cannot read");
    expect = 32 + 8LL * s->nbr_row + 8LL * (s->nbr_row - 1);
  }
  DH_CHECK(size == expect, DH_ERR_IO, "%s: %lld bytes, the state it describes takes %lld", path.c_str(), size, expect);
  return DH_OK;
}

}  // namespace dh

extern "C" {

// RealVector (per = 1) and ComplexVector (per = 2: (Re, Im) pairs) files share the header
static int write_common(const char* file_name, const double* vec, int64_t dim, int per) {
  DH_CHECK(file_name && (vec || dim == 0), DH_ERR_ARGUMENT, "null argument");
  if (dim > 0 && dh::is_device_pointer(vec)) {
    std::vector<double> host((size_t)dim * per);
    DH_CUDA(cudaMemcpy(host.data(), vec, (size_t)dim * per * sizeof(double), cudaMemcpyDeviceToHost));
    return dh::vector_file_write(file_name, host.data(), dim, per);
  }
  return dh::vector_file_write(file_name, vec, dim, per);
}

static int read_common(const char* file_name, double* vec, int64_t dim, int per) {
  DH_CHECK(file_name && (vec || dim == 0) && dim >= 0, DH_ERR_ARGUMENT, "bad argument");
  if (dim > 0 && dh::is_device_pointer(vec)) {
    std::vector<double> host((size_t)dim * per);
    int rc = dh::vector_file_read(file_name, host.data(), dim, per);
    if (rc != DH_OK) return rc;
    DH_CUDA(cudaMemcpy(vec, host.data(), (size_t)dim * per * sizeof(double), cudaMemcpyHostToDevice));
    return DH_OK;
  }
  return dh::vector_file_read(file_name, vec, dim, per);
}

int dh_vector_write(const char* file_name, const double* vec, int64_t dim) {
  return write_common(file_name, vec, dim, 1);
}

int dh_vector_file_dimension(const char* file_name, int64_t* dim) {
  DH_CHECK(file_name && dim, DH_ERR_ARGUMENT, "null argument");
  return dh::vector_file_dimension(file_name, dim, 1);
}

int dh_vector_read(const char* file_name, double* vec, int64_t dim) {
  return read_common(file_name, vec, dim, 1);
}

int dh_complex_vector_write(const char* file_name, const double* pairs, int64_t dim) {
  return write_common(file_name, pairs, dim, 2);
}

int dh_complex_vector_file_dimension(const char* file_name, int64_t* dim) {
  DH_CHECK(file_name && dim, DH_ERR_ARGUMENT, "null argument");
  return dh::vector_file_dimension(file_name, dim, 2);
}

int dh_complex_vector_read(const char* file_name, double* pairs, int64_t dim) {
  return read_common(file_name, pairs, dim, 2);
}

}  // extern "C"
