// gp_files.cpp -- the reference's particle restart and snapshot files (host code).
//
// Fortran sequential unformatted records as gfortran lays them out (record markers of
// 4 bytes, native byte order, subrecords of at most 2147483639 bytes, signs of the
// markers flagging continuation), and on top of them the two particle layouts the
// reference writes: the class restart of SAVE_PARTICLE with ISAVEPART = 2
// (save_particle.f90:116-180; read back by initiation_particle_position.f90:430-532)
// and the snapshot of PRINT_PARTICLE (print_particle.f90:145-170).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/gazpart_files.h"

struct gp_funf {
  FILE *fp;
  bool writing;
  int64_t max_sub;
  std::vector<char> buf;   // stdio buffer
};

namespace {

constexpr int64_t kChunk = int64_t(1) << 26;   // bytes per fwrite/fread call

bool write_all(FILE *fp, const void *p, int64_t n) {
  const char *c = static_cast<const char *>(p);
  while (n > 0) {
    const size_t k = (size_t)(n < kChunk ? n : kChunk);
    if (fwrite(c, 1, k, fp) != k) return false;
    c += k;
    n -= (int64_t)k;
  }
  return true;
}

bool read_all(FILE *fp, void *p, int64_t n) {
  char *c = static_cast<char *>(p);
  while (n > 0) {
    const size_t k = (size_t)(n < kChunk ? n : kChunk);
    if (fread(c, 1, k, fp) != k) return false;
    c += k;
    n -= (int64_t)k;
  }
  return true;
}

// Reads one marker: GP_OK, GP_EEOF when the file ends cleanly before it (only allowed
// at a record's head), GP_EIO when it is cut short.
int read_marker(FILE *fp, int32_t *m, bool eof_ok) {
  unsigned char b[4];
  const size_t got = fread(b, 1, 4, fp);
  if (got == 0 && eof_ok && feof(fp)) return GP_EEOF;
  if (got != 4) return GP_EIO;
  std::memcpy(m, b, 4);
  return GP_OK;
}

// Walks the subrecords of the next logical record.  With dst set, copies up to want
// bytes of its data there.  *total receives the record's length.  The stream ends
// positioned after the record unless rewind is set.
int walk_record(gp_funf *f, char *dst, int64_t want, int64_t *total, bool rewind) {
  FILE *fp = f->fp;
  const long long start = ftello(fp);
  int64_t len = 0;
  bool first = true;
  for (;;) {
    int32_t head;
    int rc = read_marker(fp, &head, first);
    if (rc) return rc;
    const int64_t n = head < 0 ? -(int64_t)head : head;
    const bool more = head < 0;
    if (dst && len < want) {
      const int64_t k = (want - len) < n ? (want - len) : n;
      if (!read_all(fp, dst + len, k)) return GP_EIO;
      if (k < n && fseeko(fp, (off_t)(n - k), SEEK_CUR) != 0) return GP_EIO;
    } else if (fseeko(fp, (off_t)n, SEEK_CUR) != 0) {
      return GP_EIO;
    }
    int32_t tail;
    rc = read_marker(fp, &tail, false);
    if (rc) return rc;
    // the tail repeats the length, negated on every subrecord but the first
    if ((tail < 0 ? -(int64_t)tail : tail) != n || (tail < 0) != !first) return GP_ERECORD;
    len += n;
    first = false;
    if (!more) break;
  }
  *total = len;
  if (rewind && fseeko(fp, (off_t)start, SEEK_SET) != 0) return GP_EIO;
  return GP_OK;
}

int write_record(gp_funf *f, const void *data, int64_t nbytes) {
  const char *c = static_cast<const char *>(data);
  int64_t left = nbytes;
  bool first = true;
  do {
    const int64_t n = left < f->max_sub ? left : f->max_sub;
    const bool more = left > n;
    const int32_t head = (int32_t)(more ? -n : n);
    const int32_t tail = (int32_t)(first ? n : -n);
    if (!write_all(f->fp, &head, 4) || !write_all(f->fp, c, n) || !write_all(f->fp, &tail, 4)) return GP_EIO;
    c += n;
    left -= n;
    first = false;
  } while (left > 0);
  return GP_OK;
}

struct FileGuard {
  gp_funf *f = nullptr;
  ~FileGuard() {
    if (f) gp_funf_close(f);
  }
  int close() {
    const int rc = gp_funf_close(f);
    f = nullptr;
    return rc;
  }
};

#define GP_FTRY(x)          \
  do {                      \
    const int rc__ = (x);   \
    if (rc__) return rc__;  \
  } while (0)

}  // namespace

extern "C" {

int gp_funf_open(const char *path, int32_t writing, gp_funf **out) {
  if (!path || !out) return GP_EBADARG;
  *out = nullptr;
  FILE *fp = fopen(path, writing ? "wb" : "rb");
  if (!fp) return GP_EIO;
  gp_funf *f = new gp_funf;
  f->fp = fp;
  f->writing = writing != 0;
  f->max_sub = GP_FUNF_MAX_SUBRECORD;
  f->buf.resize(size_t(1) << 23);
  setvbuf(fp, f->buf.data(), _IOFBF, f->buf.size());
  *out = f;
  return GP_OK;
}

int gp_funf_close(gp_funf *f) {
  if (!f) return GP_EBADARG;
  const int bad = fclose(f->fp);
  delete f;
  return bad ? GP_EIO : GP_OK;
}

int gp_funf_set_max_subrecord(gp_funf *f, int64_t nbytes) {
  if (!f || nbytes < 1 || nbytes > GP_FUNF_MAX_SUBRECORD) return GP_EBADARG;
  f->max_sub = nbytes;
  return GP_OK;
}

int gp_funf_write(gp_funf *f, const void *data, int64_t nbytes) {
  if (!f || !f->writing || nbytes < 0 || (nbytes > 0 && !data)) return GP_EBADARG;
  return write_record(f, data, nbytes);
}

int gp_funf_record_size(gp_funf *f, int64_t *nbytes) {
  if (!f || f->writing || !nbytes) return GP_EBADARG;
  return walk_record(f, nullptr, 0, nbytes, true);
}

int gp_funf_read(gp_funf *f, void *dst, int64_t nbytes) {
  if (!f || f->writing || nbytes < 0 || (nbytes > 0 && !dst)) return GP_EBADARG;
  int64_t total = 0;
  GP_FTRY(walk_record(f, static_cast<char *>(dst), nbytes, &total, false));
  return total < nbytes ? GP_ERECORD : GP_OK;
}

int gp_write_part_class(const char *path, int64_t n, int32_t polydisp, const int32_t *npclass,
                        const double *rhop, const double *emaj, double apr, const double *const *cols) {
  if (!path || n < 0 || n > INT32_MAX || polydisp < 1 || !npclass || !rhop || !emaj || !cols) return GP_EBADARG;
  for (int k = 0; k < GP_NPARTCOL; ++k)
    if (n > 0 && !cols[k]) return GP_EBADARG;
  FileGuard g;
  GP_FTRY(gp_funf_open(path, 1, &g.f));
  const int32_t npart = (int32_t)n;
  GP_FTRY(gp_funf_write(g.f, &npart, 4));
  GP_FTRY(gp_funf_write(g.f, npclass, 4 * (int64_t)polydisp));
  GP_FTRY(gp_funf_write(g.f, rhop, 8 * (int64_t)polydisp));
  GP_FTRY(gp_funf_write(g.f, emaj, 8 * (int64_t)polydisp));
  GP_FTRY(gp_funf_write(g.f, &apr, 8));
  for (int k = 0; k < GP_NPARTCOL; ++k) GP_FTRY(gp_funf_write(g.f, cols[k], 8 * n));
  return g.close();
}

int gp_read_part_class_header(const char *path, int64_t *n, int32_t *polydisp) {
  if (!path || !n || !polydisp) return GP_EBADARG;
  FileGuard g;
  GP_FTRY(gp_funf_open(path, 0, &g.f));
  int32_t npart = 0;
  GP_FTRY(gp_funf_read(g.f, &npart, 4));
  int64_t bytes = 0;
  GP_FTRY(gp_funf_record_size(g.f, &bytes));
  *n = npart;
  *polydisp = (int32_t)(bytes / 4);
  return g.close();
}

int gp_read_part_class(const char *path, int64_t n, int32_t polydisp, int32_t *npclass, double *rhop,
                       double *emaj, double *apr, double *const *cols) {
  if (!path || n < 0 || polydisp < 1 || !npclass || !rhop || !emaj || !apr || !cols) return GP_EBADARG;
  for (int k = 0; k < GP_NPARTCOL; ++k)
    if (n > 0 && !cols[k]) return GP_EBADARG;
  FileGuard g;
  GP_FTRY(gp_funf_open(path, 0, &g.f));
  int32_t npart = 0;
  GP_FTRY(gp_funf_read(g.f, &npart, 4));
  if (npart != n) return GP_EBADARG;
  GP_FTRY(gp_funf_read(g.f, npclass, 4 * (int64_t)polydisp));
  GP_FTRY(gp_funf_read(g.f, rhop, 8 * (int64_t)polydisp));
  GP_FTRY(gp_funf_read(g.f, emaj, 8 * (int64_t)polydisp));
  GP_FTRY(gp_funf_read(g.f, apr, 8));
  for (int k = 0; k < GP_NPARTCOL; ++k) GP_FTRY(gp_funf_read(g.f, cols[k], 8 * n));
  return g.close();
}

int gp_write_part_snapshot(const char *path, int64_t n, const double *const *cols) {
  if (!path || n < 0 || !cols) return GP_EBADARG;
  for (int k = 0; k < GP_NPARTCOL; ++k)
    if (n > 0 && !cols[k]) return GP_EBADARG;
  FileGuard g;
  GP_FTRY(gp_funf_open(path, 1, &g.f));
  for (int k = 0; k < GP_NPARTCOL; ++k) GP_FTRY(gp_funf_write(g.f, cols[k], 8 * n));
  return g.close();
}

int gp_read_part_snapshot(const char *path, int64_t n, double *const *cols) {
  if (!path || n < 0 || !cols) return GP_EBADARG;
  for (int k = 0; k < GP_NPARTCOL; ++k)
    if (n > 0 && !cols[k]) return GP_EBADARG;
  FileGuard g;
  GP_FTRY(gp_funf_open(path, 0, &g.f));
  for (int k = 0; k < GP_NPARTCOL; ++k) GP_FTRY(gp_funf_read(g.f, cols[k], 8 * n));
  return g.close();
}

int gp_save_part_class(gp_ctx *ctx, int32_t ig, const char *path, int32_t polydisp, const int32_t *npclass,
                       const double *rhop, const double *emaj, double apr, const int32_t *idp) {
  if (!ctx || !path || polydisp < 1 || !npclass || !rhop || !emaj) return GP_EBADARG;
  int64_t n = 0;
  GP_FTRY(gp_class_count(ctx, ig, &n));
  if (n > INT32_MAX) return GP_EBADARG;
  std::vector<double> store((size_t)n * GP_NPARTCOL);
  double *cols[GP_NPARTCOL];
  for (int k = 0; k < GP_NPARTCOL; ++k) cols[k] = store.data() + (size_t)k * n;
  if (n > 0) GP_FTRY(gp_download_class(ctx, ig, cols, 0));
  double *col_idp = cols[GP_NPARTCOL - 1];
  for (int64_t i = 0; i < n; ++i) {
    const int32_t v = idp ? idp[i] : 1;
    if (v < 1 || v > polydisp) return GP_EBADARG;
    col_idp[i] = (double)v;   // real(PART(I,J)%IDP)
  }
  return gp_write_part_class(path, n, polydisp, npclass, rhop, emaj, apr, cols);
}

int gp_load_part_class(gp_ctx *ctx, const char *path, int32_t field, int32_t *ig, int64_t *n_out) {
  if (!ctx || !path || !ig) return GP_EBADARG;
  int64_t n = 0;
  int32_t pd = 0;
  GP_FTRY(gp_read_part_class_header(path, &n, &pd));
  if (n < 0 || pd < 1) return GP_EBADARG;
  std::vector<int32_t> npclass(pd);
  std::vector<double> rhop(pd), emaj(pd), store((size_t)n * (GP_NPARTCOL + GP_NPROP));
  double apr = 0.0;
  double *cols[GP_NPARTCOL];
  for (int k = 0; k < GP_NPARTCOL; ++k) cols[k] = store.data() + (size_t)k * n;
  GP_FTRY(gp_read_part_class(path, n, pd, npclass.data(), rhop.data(), emaj.data(), &apr, cols));
  double *props[GP_NPROP];
  for (int k = 0; k < GP_NPROP; ++k) props[k] = store.data() + (size_t)(GP_NPARTCOL + k) * n;
  const double *col_idp = cols[GP_NPARTCOL - 1];
  for (int64_t i = 0; i < n; ++i) {
    const double r = col_idp[i];
    if (!(r >= 1.0 && r < (double)pd + 1.0)) return GP_EBADARG;   // int(r) in 1..pd
    const int k = (int)r - 1;
    const double a = emaj[k], b = a / apr, c = b;
    props[0][i] = a;
    props[1][i] = apr;
    props[2][i] = rhop[k];
    props[3][i] = (b * b + c * c) / 5.0;
    props[4][i] = (a * a + c * c) / 5.0;
    props[5][i] = (a * a + b * b) / 5.0;
  }
  if (n_out) *n_out = n;
  return gp_add_class(ctx, field, n, cols, props, 0, ig);
}

}  // extern "C"
