// NPY start-up and save in the reference's layout, single rank:
//   domain_init / domain_save   src/domain.c:28-86, 259-432
//   fluid_init / fluid_save     src/fluid/init.c:37-122, src/fluid/save.c:8-28
// File format: NumPy's documented .npy layout (magic, version, little-endian
// header length, dict with 'descr' / 'fortran_order' / 'shape'), dtypes
// '<f8', '<u8', '|b1' as in src/fileio.c:20-22.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <sys/stat.h>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "tcgpu.h"

extern "C" int tcgpu_report_error(const char * msg);

namespace {

int err(const std::string & m) { return tcgpu_report_error(m.c_str()); }

std::string npy_path(const char * dir, const char * name) {
  std::string d(dir);
  if (!d.empty() && d.back() != '/') d += '/';
  return d + name + ".npy";
}

// read the header; returns data offset, or 0 on failure
size_t npy_header(FILE * fp, std::string & descr, bool & fortran, std::vector<size_t> & shape) {
  unsigned char pre[12];
  if (fread(pre, 1, 8, fp) != 8 || memcmp(pre, "\x93NUMPY", 6) != 0) return 0;
  size_t hlen, prelen;
  if (pre[6] == 1) {
    if (fread(pre + 8, 1, 2, fp) != 2) return 0;
    hlen = pre[8] | (pre[9] << 8);
    prelen = 10;
  } else {
    if (fread(pre + 8, 1, 4, fp) != 4) return 0;
    hlen = (size_t)pre[8] | ((size_t)pre[9] << 8) | ((size_t)pre[10] << 16) | ((size_t)pre[11] << 24);
    prelen = 12;
  }
  std::string h(hlen, '\0');
  if (fread(&h[0], 1, hlen, fp) != hlen) return 0;
  auto value = [&](const char * key) -> size_t {
    const size_t p = h.find(std::string("'") + key + "'");
    if (p == std::string::npos) return std::string::npos;
    size_t q = h.find(':', p);
    if (q == std::string::npos) return q;
    q++;
    while (q < h.size() && h[q] == ' ') q++;
    return q;
  };
  size_t p = value("descr");
  if (p == std::string::npos || h[p] != '\'') return 0;
  const size_t e = h.find('\'', p + 1);
  descr = h.substr(p, e - p + 1);
  p = value("fortran_order");
  if (p == std::string::npos) return 0;
  fortran = h.compare(p, 4, "True") == 0;
  p = value("shape");
  if (p == std::string::npos || h[p] != '(') return 0;
  shape.clear();
  p++;
  while (p < h.size() && h[p] != ')') {
    while (p < h.size() && (h[p] == ' ' || h[p] == ',')) p++;
    if (h[p] == ')') break;
    char * end = nullptr;
    const unsigned long long v = strtoull(h.c_str() + p, &end, 10);
    if (end == h.c_str() + p) return 0;
    shape.push_back((size_t)v);
    p = (size_t)(end - h.c_str());
  }
  return prelen + hlen;
}

int npy_read(const char * dir, const char * name, const char * dtype, const std::vector<size_t> & shape,
             size_t elem, void * data) {
  const std::string path = npy_path(dir, name);
  FILE * fp = fopen(path.c_str(), "rb");
  if (!fp) return err(path + ": " + strerror(errno));
  std::string descr;
  bool fortran = false;
  std::vector<size_t> sh;
  const size_t off = npy_header(fp, descr, fortran, sh);
  if (off == 0) { fclose(fp); return err(path + ": NPY header read failed"); }
  if (descr != dtype) { fclose(fp); return err(path + ": dtype " + descr + ", " + dtype + " expected"); }
  if (fortran) { fclose(fp); return err(path + ": fortran order is not supported"); }
  if (sh != shape) { fclose(fp); return err(path + ": shape mismatch"); }
  size_t n = 1;
  for (size_t s : shape) n *= s;
  const size_t got = fread(data, elem, n, fp);
  fclose(fp);
  if (got != n) return err(path + ": short read");
  return 0;
}

int npy_write(const char * dir, const char * name, const char * dtype, const std::vector<size_t> & shape,
              size_t elem, const void * data) {
  const std::string path = npy_path(dir, name);
  std::string d = std::string("{'descr': ") + dtype + ", 'fortran_order': False, 'shape': (";
  for (size_t i = 0; i < shape.size(); i++) {
    d += std::to_string(shape[i]);
    if (shape.size() == 1) d += ",";
    else if (i + 1 < shape.size()) d += ", ";
  }
  d += "), }";
  size_t total = 10 + d.size() + 1;
  const size_t padded = (total + 63) / 64 * 64;
  d.append(padded - total, ' ');
  d += '\n';
  const size_t hlen = d.size();
  unsigned char pre[10] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0, (unsigned char)(hlen & 0xff), (unsigned char)(hlen >> 8)};
  FILE * fp = fopen(path.c_str(), "wb");
  if (!fp) return err(path + ": " + strerror(errno));
  size_t n = 1;
  for (size_t s : shape) n *= s;
  const bool ok = fwrite(pre, 1, 10, fp) == 10 && fwrite(d.data(), 1, hlen, fp) == hlen && fwrite(data, elem, n, fp) == n;
  fclose(fp);
  if (!ok) return err(path + ": write failed");
  return 0;
}

double * dcalloc(size_t n) { return static_cast<double *>(calloc(n > 0 ? n : 1, sizeof(double))); }

int prepare(const domain_t * d, const int nadds[3][2], array_t * a) {
  size_t n = 1;
  for (int dim = 0; dim < 3; dim++) n *= d->mysizes[dim] + nadds[dim][0] + nadds[dim][1];
  a->size = sizeof(double);
  a->nadds = static_cast<int (*)[2]>(calloc(3, 2 * sizeof(int)));
  for (int dim = 0; dim < 3; dim++) {
    a->nadds[dim][0] = nadds[dim][0];
    a->nadds[dim][1] = nadds[dim][1];
  }
  a->datasize = n * sizeof(double);
  a->data = calloc(n, sizeof(double));
  if (a->nadds == nullptr || a->data == nullptr) return err("memory allocation failed");
  return 0;
}

// array.c:124-152: the file holds x with its additional cells, y and z without
int load_field(const domain_t * d, const char * dir, const char * name, array_t * a) {
  const size_t nx = d->glsizes[0], ny = d->glsizes[1], nz = d->glsizes[2];
  const int ax = a->nadds[0][0] + a->nadds[0][1];
  const size_t rowlen = nx + ax;
  std::vector<double> buf(rowlen * ny * nz);
  if (npy_read(dir, name, "'<f8'", {nz, ny, rowlen}, sizeof(double), buf.data())) return 1;
  double * dst = static_cast<double *>(a->data);
  for (size_t k = 0; k < nz; k++)
    for (size_t j = 0; j < ny; j++)
      memcpy(dst + rowlen * ((j + 1) + (ny + 2) * (k + 1)), buf.data() + rowlen * (j + ny * k), rowlen * sizeof(double));
  return 0;
}

int save_field(const domain_t * d, const char * dir, const char * name, const array_t * a) {
  const size_t nx = d->glsizes[0], ny = d->glsizes[1], nz = d->glsizes[2];
  const int ax = a->nadds[0][0] + a->nadds[0][1];
  const size_t rowlen = nx + ax;
  std::vector<double> buf(rowlen * ny * nz);
  const double * src = static_cast<const double *>(a->data);
  for (size_t k = 0; k < nz; k++)
    for (size_t j = 0; j < ny; j++)
      memcpy(buf.data() + rowlen * (j + ny * k), src + rowlen * ((j + 1) + (ny + 2) * (k + 1)), rowlen * sizeof(double));
  return npy_write(dir, name, "'<f8'", {nz, ny, rowlen}, sizeof(double), buf.data());
}

}  // namespace

extern "C" {

int domain_init(const char dirname_ic[], domain_t * domain) {
  if (domain == nullptr || dirname_ic == nullptr) return err("domain_init: NULL argument");
  bool is_curved = false;
  if (npy_read(dirname_ic, "is_curved", "'|b1'", {}, sizeof(bool), &is_curved)) return 1;
  size_t gl[3];
  if (npy_read(dirname_ic, "glsizes", "'<u8'", {3}, sizeof(size_t), gl)) return 1;
  double len[3];
  if (npy_read(dirname_ic, "lengths", "'<f8'", {3}, sizeof(double), len)) return 1;
  const size_t nx = gl[0], ny = gl[1], nz = gl[2];
  double * xf = dcalloc(nx + 1);
  double * xc = dcalloc(nx + 2);
  if (npy_read(dirname_ic, "xf", "'<f8'", {nx + 1}, sizeof(double), xf)) return 1;
  if (npy_read(dirname_ic, "xc", "'<f8'", {nx + 2}, sizeof(double), xc)) return 1;
  domain->info = nullptr;
  domain->is_curved = is_curved;
  for (int d = 0; d < 3; d++) {
    domain->glsizes[d] = gl[d];
    domain->mysizes[d] = gl[d];
    domain->offsets[d] = 0;
    domain->lengths[d] = len[d];
  }
  domain->xf = xf;
  domain->xc = xc;
  // XF(I) = xf[I-1], XC(I) = xc[I], HXXF(I) = hxxf[I-1], HXXC(I) = hxxc[I], ...
  double * hxxf = dcalloc(nx + 1);
  double * hxxc = dcalloc(nx + 2);
  double * hyxf = dcalloc(nx + 1);
  double * hyxc = dcalloc(nx + 2);
  double * jdxf = dcalloc(nx + 1);
  double * jdxc = dcalloc(nx + 2);
  for (size_t i = 1; i <= nx + 1; i++) hxxf[i - 1] = xc[i] - xc[i - 1];
  hxxc[0] = 0.5 * xf[1] - 0.5 * xf[0];
  for (size_t i = 1; i <= nx; i++) hxxc[i] = xf[i] - xf[i - 1];
  hxxc[nx + 1] = 0.5 * xf[nx] - 0.5 * xf[nx - 1];
  const double ly = len[1];
  for (size_t i = 1; i <= nx + 1; i++) hyxf[i - 1] = is_curved ? xf[i - 1] * ly / ny : ly / ny;
  for (size_t i = 0; i <= nx + 1; i++) hyxc[i] = is_curved ? xc[i] * ly / ny : ly / ny;
  const double hz = len[2] / nz;
  for (size_t i = 1; i <= nx + 1; i++) jdxf[i - 1] = hxxf[i - 1] * hyxf[i - 1] * hz;
  for (size_t i = 0; i <= nx + 1; i++) jdxc[i] = hxxc[i] * hyxc[i] * hz;
  domain->hxxf = hxxf;
  domain->hxxc = hxxc;
  domain->hyxf = hyxf;
  domain->hyxc = hyxc;
  domain->jdxf = jdxf;
  domain->jdxc = jdxc;
  domain->hz = hz;
  return 0;
}

int domain_save(const char dirname[], const domain_t * domain) {
  const size_t nx = domain->glsizes[0];
  const bool is_curved = domain->is_curved;
  if (npy_write(dirname, "is_curved", "'|b1'", {}, sizeof(bool), &is_curved)) return 1;
  if (npy_write(dirname, "glsizes", "'<u8'", {3}, sizeof(size_t), domain->glsizes)) return 1;
  if (npy_write(dirname, "lengths", "'<f8'", {3}, sizeof(double), domain->lengths)) return 1;
  if (npy_write(dirname, "xf", "'<f8'", {nx + 1}, sizeof(double), domain->xf)) return 1;
  if (npy_write(dirname, "xc", "'<f8'", {nx + 2}, sizeof(double), domain->xc)) return 1;
  return 0;
}

// the host arrays of fluid_t (src/fluid/init.c:42-68) and Re, Pr from the
// environment (:112-122); shared by fluid_init and the device-generated
// initial field
__attribute__((visibility("hidden"))) int tcgpu_io_fluid_alloc(const domain_t * domain, fluid_t * fluid);

int fluid_init(const char dirname_ic[], const domain_t * domain, fluid_t * fluid) {
  if (domain == nullptr || fluid == nullptr) return err("fluid_init: NULL argument");
  if (tcgpu_io_fluid_alloc(domain, fluid)) return 1;
  if (load_field(domain, dirname_ic, "ux", &fluid->ux) || load_field(domain, dirname_ic, "uy", &fluid->uy) ||
      load_field(domain, dirname_ic, "uz", &fluid->uz) || load_field(domain, dirname_ic, "p", &fluid->p) ||
      load_field(domain, dirname_ic, "t", &fluid->t))
    return 1;
  if (fluid_update_boundaries_ux(domain, &fluid->ux) || fluid_update_boundaries_uy(domain, &fluid->uy) ||
      fluid_update_boundaries_uz(domain, &fluid->uz) || fluid_update_boundaries_p(domain, &fluid->p) ||
      fluid_update_boundaries_t(domain, &fluid->t))
    return 1;
  return 0;
}

__attribute__((visibility("hidden"))) int tcgpu_io_fluid_alloc(const domain_t * domain, fluid_t * fluid) {
  if (domain == nullptr || fluid == nullptr) return err("fluid_init: NULL argument");
  // array_macros/fluid/*.h NADDS
  static const int C[3][2] = {{1, 1}, {1, 1}, {1, 1}};
  static const int F[3][2] = {{0, 1}, {1, 1}, {1, 1}};
  static const int TF[3][2] = {{0, 1}, {1, 1}, {1, 1}};
  static const int TC[3][2] = {{0, 0}, {1, 1}, {1, 1}};
  static const int SX[3][2] = {{-1, 0}, {0, 0}, {0, 0}};
  static const int SC[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  if (prepare(domain, F, &fluid->ux) || prepare(domain, C, &fluid->uy) || prepare(domain, C, &fluid->uz) ||
      prepare(domain, C, &fluid->p) || prepare(domain, C, &fluid->psi) || prepare(domain, C, &fluid->t))
    return 1;
  if (prepare(domain, TC, &fluid->lxx) || prepare(domain, TF, &fluid->lyx0) || prepare(domain, TF, &fluid->lyx1) ||
      prepare(domain, TF, &fluid->lzx) || prepare(domain, TF, &fluid->lxy) || prepare(domain, TC, &fluid->lyy0) ||
      prepare(domain, TC, &fluid->lyy1) || prepare(domain, TC, &fluid->lzy) || prepare(domain, TF, &fluid->lxz) ||
      prepare(domain, TC, &fluid->lyz) || prepare(domain, TC, &fluid->lzz))
    return 1;
  for (int n = 0; n < 3; n++) {
    if (prepare(domain, SX, &fluid->srcux[n]) || prepare(domain, SC, &fluid->srcuy[n]) ||
        prepare(domain, SC, &fluid->srcuz[n]) || prepare(domain, SC, &fluid->srct[n]))
      return 1;
  }
  const char * names[2] = {"Re", "Pr"};
  double * dst[2] = {&fluid->Re, &fluid->Pr};
  for (int n = 0; n < 2; n++) {
    const char * s = getenv(names[n]);
    if (s == nullptr) return err(std::string(names[n]) + " not found");
    errno = 0;
    *dst[n] = strtod(s, nullptr);
    if (errno != 0) return err(std::string(names[n]) + ": invalid value as double");
  }
  return 0;
}

// The statistics directory of src/statistics.c:250-300: num, the domain, and
// the eight accumulators as (nz, ny, nx + 1) or (nz, ny, nx + 2) arrays in the
// order ux1 ux2 uy1 uy2 uz1 uz2 adv dif (array.c:155-222 writes the interior
// j, k with x's additional cells, which is the device layout as it is). As in
// the reference, a directory that cannot be created is not an error by itself.
__attribute__((visibility("hidden"))) int tcgpu_io_write_statistics(const char dirname[], const domain_t * domain,
                                                                    size_t num, const double * const arrays[8]) {
  mkdir(dirname, 0755);
  if (npy_write(dirname, "num", "'<u8'", {}, sizeof(size_t), &num)) return 1;
  if (domain_save(dirname, domain)) return 1;
  const size_t nx = domain->glsizes[0], ny = domain->glsizes[1], nz = domain->glsizes[2];
  static const char * names[8] = {"ux1", "ux2", "uy1", "uy2", "uz1", "uz2", "adv", "dif"};
  for (int s = 0; s < 8; s++) {
    const size_t rowlen = (s >= 2 && s <= 5) ? nx + 2 : nx + 1;
    if (npy_write(dirname, names[s], "'<f8'", {nz, ny, rowlen}, sizeof(double), arrays[s])) return 1;
  }
  return 0;
}

int fluid_save(const char dirname[], const domain_t * domain, const fluid_t * fluid) {
  if (npy_write(dirname, "Re", "'<f8'", {}, sizeof(double), &fluid->Re)) return 1;
  if (npy_write(dirname, "Pr", "'<f8'", {}, sizeof(double), &fluid->Pr)) return 1;
  if (save_field(domain, dirname, "ux", &fluid->ux) || save_field(domain, dirname, "uy", &fluid->uy) ||
      save_field(domain, dirname, "uz", &fluid->uz) || save_field(domain, dirname, "p", &fluid->p) ||
      save_field(domain, dirname, "t", &fluid->t))
    return 1;
  return 0;
}

}  // extern "C"
