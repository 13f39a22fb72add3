// io.cu -- on-disk formats of the reference's writers and readers (host code;
// see io.h for the format rules and the reference files they follow).
#include <fcntl.h>
#include <stdint.h>
#include <stdio.h>
#include <sys/types.h>
#include <unistd.h>
#include <string.h>

#include <string>
#include <vector>

#include "io.h"
#include "openpfc_b200.h"

namespace opfc {
namespace io {

namespace {

bool is_flag(char c) { return c == '-' || c == '+' || c == ' ' || c == '0'; }
bool is_digit(char c) { return c >= '0' && c <= '9'; }

// Position of the single valid "%[flags][*][width]d", or -1 (err set).
int find_spec(const char *p, size_t &spec_len, std::string &err) {
  int at = -1;
  for (size_t i = 0; p[i]; ++i) {
    if (p[i] != '%') continue;
    if (at >= 0) {
      err = "format_with_number: invalid filename pattern (more than one '%')";
      return -2;
    }
    size_t k = i + 1;
    while (is_flag(p[k])) ++k;
    if (p[k] == '*') ++k;
    while (is_digit(p[k])) ++k;
    if (p[k] != 'd') {
      err = "format_with_number: invalid filename pattern: only one %d integer specifier "
            "(optional flags -+ 0, width) is allowed";
      return -2;
    }
    at = (int)i;
    spec_len = k + 1 - i;
    i = k;
  }
  return at;
}

}  // namespace

int format_with_number(const char *pattern, int increment, std::string &out, std::string &err) {
  if (!pattern) {
    err = "format_with_number: null pattern";
    return OPFC_ERR_ARG;
  }
  size_t len = 0;
  const int at = find_spec(pattern, len, err);
  if (at == -2) return OPFC_ERR_ARG;
  if (at < 0) {
    out = pattern;
    return OPFC_OK;
  }
  std::string spec(pattern + at, len);
  const bool star = spec.find('*') != std::string::npos;
  char buf[64];
  // '*' takes the width from the argument list, as the reference's
  // string_format(filename, increment) does: the increment is the width and
  // the value is undefined there; here the value 0 is printed in that width.
  const int n = star ? snprintf(buf, sizeof buf, spec.c_str(), increment, 0)
                     : snprintf(buf, sizeof buf, spec.c_str(), increment);
  if (n < 0 || n >= (int)sizeof buf) {
    err = "format_with_number: formatted number too long";
    return OPFC_ERR_ARG;
  }
  out.assign(pattern, at);
  out += buf;
  out += pattern + at + len;
  return OPFC_OK;
}

namespace {
// pwrite all of `bytes` at `at`
bool pwrite_all(int fd, const void *p, size_t bytes, off_t at) {
  const char *c = static_cast<const char *>(p);
  while (bytes) {
    const ssize_t w = pwrite(fd, c, bytes, at);
    if (w <= 0) return false;
    c += w;
    bytes -= (size_t)w;
    at += w;
  }
  return true;
}
}  // namespace

int write_box(const std::string &fn, const int global[3], const int local[3], const int offset[3],
              const double *data, int ncomp, std::string &err) {
  // The whole array truncates the file first (the reference's collective
  // MPI_File_set_size(fh, 0) before MPI_File_write_all).  A smaller box is
  // written in place, creating the file if it is missing but never truncating
  // it, so several writers can each fill their own box of one file; the
  // coordinator truncates and sizes the file once beforehand (prepare_box_file).
  const bool whole = local[0] == global[0] && local[1] == global[1] && local[2] == global[2];
  const int fd = open(fn.c_str(), O_WRONLY | O_CREAT | (whole ? O_TRUNC : 0), 0666);
  if (fd < 0) {
    err = "cannot open \"" + fn + "\" for writing";
    return OPFC_ERR_IO;
  }
  const size_t row = (size_t)local[0] * ncomp;
  bool ok = true;
  if (whole) {
    ok = pwrite_all(fd, data, row * local[1] * local[2] * sizeof(double), 0);
  } else {
    for (int k = 0; k < local[2] && ok; ++k)
      for (int j = 0; j < local[1] && ok; ++j) {
        const long long at =
            ((long long)(offset[2] + k) * global[1] + (offset[1] + j)) * global[0] + offset[0];
        ok = pwrite_all(fd, data + ((size_t)k * local[1] + j) * row, row * sizeof(double),
                        (off_t)(at * ncomp * (long long)sizeof(double)));
      }
  }
  ok = (close(fd) == 0) && ok;
  if (!ok) {
    err = "short write to \"" + fn + "\"";
    return OPFC_ERR_IO;
  }
  return OPFC_OK;
}

int prepare_box_file(const std::string &fn, const int global[3], int ncomp, std::string &err) {
  const int fd = open(fn.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0666);
  if (fd < 0) {
    err = "cannot open \"" + fn + "\" for writing";
    return OPFC_ERR_IO;
  }
  const off_t bytes = (off_t)global[0] * global[1] * global[2] * ncomp * (off_t)sizeof(double);
  const bool ok = ftruncate(fd, bytes) == 0;
  if (close(fd) != 0 || !ok) {
    err = "cannot size \"" + fn + "\"";
    return OPFC_ERR_IO;
  }
  return OPFC_OK;
}

int read_box(const std::string &fn, const int global[3], const int local[3], const int offset[3], double *data,
             int ncomp, std::string &err) {
  FILE *f = fopen(fn.c_str(), "rb");
  if (!f) {
    err = "cannot open \"" + fn + "\" for reading";
    return OPFC_ERR_IO;
  }
  const size_t row = (size_t)local[0] * ncomp;
  bool ok = true;
  for (int k = 0; k < local[2] && ok; ++k)
    for (int j = 0; j < local[1] && ok; ++j) {
      const long long at = ((long long)(offset[2] + k) * global[1] + (offset[1] + j)) * global[0] + offset[0];
      ok = fseeko(f, (off_t)(at * ncomp * (long long)sizeof(double)), SEEK_SET) == 0 &&
           fread(data + ((size_t)k * local[1] + j) * row, sizeof(double), row, f) == row;
    }
  fclose(f);
  if (!ok) {
    err = "\"" + fn + "\" holds fewer values than the domain needs";
    return OPFC_ERR_SIZE;
  }
  return OPFC_OK;
}

int write_vti(const std::string &fn, const int global[3], const int local[3], const int offset[3],
              const double origin[3], const double spacing[3], const char *name, const double *data,
              std::string &err) {
  FILE *f = fopen(fn.c_str(), "wb");
  if (!f) {
    err = "cannot open \"" + fn + "\" for writing";
    return OPFC_ERR_IO;
  }
  fprintf(f, "<?xml version=\"1.0\" encoding=\"utf-8\"?>\n");
  fprintf(f, "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n");
  fprintf(f, "  <ImageData WholeExtent=\"0 %d 0 %d 0 %d\" Origin=\"%g %g %g\" Spacing=\"%g %g %g\">\n",
          global[0] - 1, global[1] - 1, global[2] - 1, origin[0], origin[1], origin[2], spacing[0], spacing[1],
          spacing[2]);
  fprintf(f, "    <Piece Extent=\"%d %d %d %d %d %d\">\n", offset[0], offset[0] + local[0] - 1, offset[1],
          offset[1] + local[1] - 1, offset[2], offset[2] + local[2] - 1);
  fprintf(f, "      <PointData>\n");
  fprintf(f, "        <DataArray type=\"Float64\" Name=\"%s\" NumberOfComponents=\"1\" format=\"appended\" offset=\"0\"/>\n",
          name ? name : "Field");
  fprintf(f, "      </PointData>\n");
  fprintf(f, "    </Piece>\n");
  fprintf(f, "  </ImageData>\n");
  fprintf(f, "  <AppendedData encoding=\"raw\">\n");
  fputc('_', f);
  const size_t count = (size_t)local[0] * local[1] * local[2];
  const uint64_t bytes = (uint64_t)count * sizeof(double);
  bool ok = fwrite(&bytes, sizeof bytes, 1, f) == 1 && fwrite(data, sizeof(double), count, f) == count;
  fprintf(f, "\n  </AppendedData>\n</VTKFile>\n");
  ok = (fclose(f) == 0) && ok;
  if (!ok) {
    err = "short write to \"" + fn + "\"";
    return OPFC_ERR_IO;
  }
  return OPFC_OK;
}

}  // namespace io
}  // namespace opfc

extern "C" int opfc_format_filename(const char *pattern, int increment, char *out, size_t out_len) {
  std::string s, err;
  const int rc = opfc::io::format_with_number(pattern, increment, s, err);
  if (rc) return rc;
  if (!out || s.size() + 1 > out_len) return OPFC_ERR_SIZE;
  memcpy(out, s.c_str(), s.size() + 1);
  return OPFC_OK;
}

namespace {
bool box_ok(const int g[3], const int l[3], const int o[3]) {
  if (!g || !l || !o) return false;
  for (int a = 0; a < 3; ++a)
    if (g[a] < 1 || l[a] < 1 || o[a] < 0 || o[a] + l[a] > g[a]) return false;
  return true;
}
}  // namespace

extern "C" int opfc_write_raw(const char *filename, const int global[3], const int local[3], const int offset[3],
                              const double *data, int ncomp) {
  if (!filename || !data || (ncomp != 1 && ncomp != 2) || !box_ok(global, local, offset)) return OPFC_ERR_ARG;
  std::string err;
  return opfc::io::write_box(filename, global, local, offset, data, ncomp, err);
}

extern "C" int opfc_prepare_raw(const char *filename, const int global[3], int ncomp) {
  const int origin[3] = {0, 0, 0};
  if (!filename || (ncomp != 1 && ncomp != 2) || !box_ok(global, global, origin)) return OPFC_ERR_ARG;
  std::string err;
  return opfc::io::prepare_box_file(filename, global, ncomp, err);
}

extern "C" int opfc_read_raw(const char *filename, const int global[3], const int local[3], const int offset[3],
                             double *data, int ncomp) {
  if (!filename || !data || (ncomp != 1 && ncomp != 2) || !box_ok(global, local, offset)) return OPFC_ERR_ARG;
  std::string err;
  return opfc::io::read_box(filename, global, local, offset, data, ncomp, err);
}

extern "C" int opfc_write_vti_raw(const char *filename, const int global[3], const int local[3],
                                  const int offset[3], const double origin[3], const double spacing[3],
                                  const char *name, const double *data) {
  if (!filename || !data || !origin || !spacing || !box_ok(global, local, offset)) return OPFC_ERR_ARG;
  std::string err;
  return opfc::io::write_vti(filename, global, local, offset, origin, spacing, name, data, err);
}
