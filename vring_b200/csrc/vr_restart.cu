// vr_restart.cu -- restart files of run.F90:390-539 (restart_save /
// restart_load) and their extension for exact resumes.
//
// The reference writes gfortran unformatted sequential records: each payload
// framed by its length as a 4-byte little-endian integer before and after.
// File layout (one rank): a header record (nstep int32, ntime real64,
// nthetag, nrg, nzg int32), then for iz = 1..nz, ir = 1..nr, ith = 1..ntheta
// one record (q1, q2, q3) of the interior cell.  That file restarts a run
// only approximately: ghosts, pressure, the pressure gradient, the RK history
// and the outflow state are not in it.
//
// vr_restart_save(.., VR_RESTART_FULL) appends, after the reference's
// records, an extension the reference's reader never reaches (it closes the
// file after the q records): a tagged header record with the clock, then
// every field of the context in its full ghosted layout.  vr_restart_load
// reads the reference part and, when the extension follows, the whole state,
// so a resumed run continues bit for bit.  The particle classes have their
// own file (vr_part_restart_save / _load).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "vr_internal.cuh"

namespace {

const char kExtMagic[8] = {'V', 'R', 'B', '2', 'R', 'S', 'T', '1'};

struct File {
  FILE *f = nullptr;
  explicit File(const char *path, const char *mode) { f = std::fopen(path, mode); }
  ~File() {
    if (f) std::fclose(f);
  }
  bool close() {
    bool ok = std::fclose(f) == 0;
    f = nullptr;
    return ok;
  }
};

}  // namespace

namespace vr {

bool rec_write(FILE *f, const void *buf, size_t n) {
  if (n > 0x7fffffffu) return false;
  const int32_t m = (int32_t)n;
  return std::fwrite(&m, 4, 1, f) == 1 && std::fwrite(buf, 1, n, f) == n && std::fwrite(&m, 4, 1, f) == 1;
}

// reads one record of exactly n bytes
bool rec_read(FILE *f, void *buf, size_t n) {
  int32_t a = 0, b = 0;
  if (std::fread(&a, 4, 1, f) != 1 || (size_t)a != n) return false;
  if (std::fread(buf, 1, n, f) != n) return false;
  return std::fread(&b, 4, 1, f) == 1 && (size_t)b == n;
}

constexpr size_t kChunkDoubles = (size_t)1 << 24;  // 128 MiB per data record

bool data_write(FILE *f, const double *p, size_t n) {
  for (size_t o = 0; o < n; o += kChunkDoubles)
    if (!rec_write(f, p + o, sizeof(double) * std::min(kChunkDoubles, n - o))) return false;
  return true;
}

bool data_read(FILE *f, double *p, size_t n) {
  for (size_t o = 0; o < n; o += kChunkDoubles)
    if (!rec_read(f, p + o, sizeof(double) * std::min(kChunkDoubles, n - o))) return false;
  return true;
}

}  // namespace vr

namespace {

// the fields of a context, in the order of the extension
const int32_t kFields[] = {VR_F_Q1,   VR_F_Q2,   VR_F_Q3,    VR_F_DQ1,    VR_F_DQ2,   VR_F_DQ3,
                           VR_F_RU1,  VR_F_RU2,  VR_F_RU3,   VR_F_PRES,   VR_F_PRG,   VR_F_RHS,
                           VR_F_DPH,  VR_F_DQ3NO, VR_F_CORR3S, VR_F_CORR3N, VR_F_CSORT, VR_F_TCONV};

size_t count(const int64_t e[4]) { return (size_t)e[0] * e[1] * e[2] * e[3]; }

}  // namespace

using namespace vr;

extern "C" int vr_restart_save(vr_ctx *c, const char *path, int32_t flags) {
  if (!c || !path) return VR_ERR_ARG;
  const Geo &g = c->geo;
  int64_t ext[4];
  int rc = vr_field_extents(c, VR_F_Q1, ext);
  if (rc) return rc;
  const size_t n = count(ext);
  std::vector<double> q[3];
  for (int m = 0; m < 3; m++) {
    q[m].resize(n);
    if ((rc = vr_get_field(c, VR_F_Q1 + m, q[m].data(), ext))) return rc;
  }
  File F(path, "wb");
  if (!F.f) return set_err(c, VR_ERR_IO, std::string("cannot open ") + path);
  unsigned char h[24];
  const int32_t nstep = (int32_t)c->nstep, nth = g.nth, nr = g.nr, nz = g.nz;
  std::memcpy(h, &nstep, 4);
  std::memcpy(h + 4, &c->ntime, 8);
  std::memcpy(h + 12, &nth, 4);
  std::memcpy(h + 16, &nr, 4);
  std::memcpy(h + 20, &nz, 4);
  bool ok = rec_write(F.f, h, 24);
  // one z plane of records at a time: [len][q1 q2 q3][len] per cell
  std::vector<unsigned char> plane((size_t)nr * nth * 32);
  for (int iz = 1; iz <= nz && ok; iz++) {
    unsigned char *b = plane.data();
    for (int ir = 1; ir <= nr; ir++)
      for (int ith = 1; ith <= nth; ith++) {
        const size_t o = (size_t)I3(g, ith, ir, iz);
        const int32_t m = 24;
        const double v[3] = {q[0][o], q[1][o], q[2][o]};
        std::memcpy(b, &m, 4);
        std::memcpy(b + 4, v, 24);
        std::memcpy(b + 28, &m, 4);
        b += 32;
      }
    ok = std::fwrite(plane.data(), 1, plane.size(), F.f) == plane.size();
  }
  if (ok && (flags & VR_RESTART_FULL)) {
    // extension: magic, version, clock, field count; then per field its id
    // and extents and its data in the context's layout
    unsigned char x[8 + 4 + 4 + 8 + 8 + 4];
    const int32_t ver = 1, irk = c->irk, nf = (int32_t)(sizeof(kFields) / sizeof(kFields[0]));
    const int64_t ns = c->nstep;
    std::memcpy(x, kExtMagic, 8);
    std::memcpy(x + 8, &ver, 4);
    std::memcpy(x + 12, &irk, 4);
    std::memcpy(x + 16, &ns, 8);
    std::memcpy(x + 24, &c->ntime, 8);
    std::memcpy(x + 32, &nf, 4);
    ok = rec_write(F.f, x, sizeof(x));
    std::vector<double> buf;
    for (int32_t id : kFields) {
      if (!ok) break;
      int64_t e[4];
      if ((rc = vr_field_extents(c, id, e))) return rc;
      buf.resize(count(e));
      if ((rc = vr_get_field(c, id, buf.data(), e))) return rc;
      unsigned char fh[4 + 32];
      std::memcpy(fh, &id, 4);
      std::memcpy(fh + 4, e, 32);
      ok = rec_write(F.f, fh, sizeof(fh)) && data_write(F.f, buf.data(), buf.size());
    }
  }
  if (!ok || !F.close()) return set_err(c, VR_ERR_IO, std::string("write failed: ") + path);
  return VR_OK;
}

extern "C" int vr_restart_load(vr_ctx *c, const char *path, int32_t *full) {
  if (!c || !path) return VR_ERR_ARG;
  if (full) *full = 0;
  const Geo &g = c->geo;
  File F(path, "rb");
  if (!F.f) return set_err(c, VR_ERR_IO, std::string("cannot open ") + path);
  unsigned char h[24];
  if (!rec_read(F.f, h, 24)) return set_err(c, VR_ERR_IO, "restart header record");
  int32_t nstep, nth, nr, nz;
  double ntime;
  std::memcpy(&nstep, h, 4);
  std::memcpy(&ntime, h + 4, 8);
  std::memcpy(&nth, h + 12, 4);
  std::memcpy(&nr, h + 16, 4);
  std::memcpy(&nz, h + 20, 4);
  if (nth != g.nth || nr != g.nr || nz != g.nz)
    return set_err(c, VR_ERR_FIELD, "restart grid " + std::to_string(nth) + "x" + std::to_string(nr) + "x" +
                                        std::to_string(nz) + " differs from the context");
  int64_t ext[4];
  int rc = vr_field_extents(c, VR_F_Q1, ext);
  if (rc) return rc;
  const size_t n = count(ext);
  std::vector<double> q[3];
  for (int m = 0; m < 3; m++) {
    q[m].resize(n);
    if ((rc = vr_get_field(c, VR_F_Q1 + m, q[m].data(), ext))) return rc;
  }
  std::vector<unsigned char> plane((size_t)nr * nth * 32);
  for (int iz = 1; iz <= nz; iz++) {
    if (std::fread(plane.data(), 1, plane.size(), F.f) != plane.size())
      return set_err(c, VR_ERR_IO, "restart: file ends inside the q records");
    const unsigned char *b = plane.data();
    for (int ir = 1; ir <= nr; ir++)
      for (int ith = 1; ith <= nth; ith++) {
        int32_t a, e;
        std::memcpy(&a, b, 4);
        std::memcpy(&e, b + 28, 4);
        if (a != 24 || e != 24) return set_err(c, VR_ERR_IO, "restart: bad record marker in the q records");
        const size_t o = (size_t)I3(g, ith, ir, iz);
        std::memcpy(&q[0][o], b + 4, 8);
        std::memcpy(&q[1][o], b + 12, 8);
        std::memcpy(&q[2][o], b + 20, 8);
        b += 32;
      }
  }
  for (int m = 0; m < 3; m++)
    if ((rc = vr_set_field(c, VR_F_Q1 + m, q[m].data(), ext))) return rc;
  c->nstep = nstep;  // the reference's nstepi
  c->ntime = ntime;
  // the extension, when present
  int32_t m0 = 0;
  if (std::fread(&m0, 4, 1, F.f) != 1) return VR_OK;  // reference file: done
  unsigned char x[8 + 4 + 4 + 8 + 8 + 4];
  if (m0 != (int32_t)sizeof(x) || std::fread(x, 1, sizeof(x), F.f) != sizeof(x) || std::memcmp(x, kExtMagic, 8))
    return set_err(c, VR_ERR_IO, "restart: unknown data after the q records");
  int32_t m1 = 0;
  if (std::fread(&m1, 4, 1, F.f) != 1 || m1 != m0) return set_err(c, VR_ERR_IO, "restart: extension header");
  int32_t ver, irk, nf;
  int64_t ns;
  double nt;
  std::memcpy(&ver, x + 8, 4);
  std::memcpy(&irk, x + 12, 4);
  std::memcpy(&ns, x + 16, 8);
  std::memcpy(&nt, x + 24, 8);
  std::memcpy(&nf, x + 32, 4);
  if (ver != 1 || nf < 0 || nf > 64) return set_err(c, VR_ERR_IO, "restart: extension version");
  std::vector<double> buf;
  for (int i = 0; i < nf; i++) {
    unsigned char fh[4 + 32];
    if (!rec_read(F.f, fh, sizeof(fh))) return set_err(c, VR_ERR_IO, "restart: field header");
    int32_t id;
    int64_t e[4], want[4];
    std::memcpy(&id, fh, 4);
    std::memcpy(e, fh + 4, 32);
    if ((rc = vr_field_extents(c, id, want))) return rc;
    if (std::memcmp(e, want, sizeof(e))) return set_err(c, VR_ERR_FIELD, "restart: field extents differ");
    buf.resize(count(e));
    if (!data_read(F.f, buf.data(), buf.size())) return set_err(c, VR_ERR_IO, "restart: field data");
    if ((rc = vr_set_field(c, id, buf.data(), e))) return rc;
  }
  if (irk < 1 || irk > 3) return set_err(c, VR_ERR_IO, "restart: substep out of range");
  c->irk = irk;
  c->nstep = ns;
  c->ntime = nt;
  if (full) *full = 1;
  return VR_OK;
}
