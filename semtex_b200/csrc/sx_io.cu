// sx_io.cu -- field files in the reference's format and compare-style norms.
//
// A field file is a 10-line ASCII header followed by binary data.  Header
// lines, each a left-justified value then its label (the Header writer,
// src/data2df.cpp:503-535, and the readers strm>>Domain,
// src/domain.cpp:284-400, and compare, utility/compare.cpp:112-175):
//   session                          Session
//   creation date                    Created
//   np np nz nel                     Nr, Ns, Nz, Elements
//   step                             Step
//   time                             Time
//   time step                        Time step
//   kinematic viscosity              Kinvis
//   beta                             Beta
//   one character per field          Fields written
//   "binary IEEE little-endian"      Format
// Data: field after field, plane after plane, the nel np np values of each
// plane (ostream<<AuxField, src/auxfield.cpp:997-1040); a reader byte-swaps
// when the file's endianness differs from the machine's and zeroes the
// padding of each plane (istream>>AuxField, src/auxfield.cpp:1043-1095).
//
// Norms (GPU): compare's inf-norm of exact - computed over all planes
// (utility/compare.cpp:206-218) and, per plane, AuxField::errors' L2 figure
// (src/auxfield.cpp:813-860: each element's sqrt(sum e^2 Q4), summed, over
// the summed element areas), at the fields' own GLL points.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <string>
#include <utility>
#include <vector>

#include "sx_modal.h"

using namespace sx;

namespace {

bool host_little_endian() {
  const uint16_t v = 1;
  unsigned char c;
  std::memcpy(&c, &v, 1);
  return c == 1;
}

void swap8(double *p, size_t n) {
  for (size_t i = 0; i < n; i++) {
    unsigned char *c = reinterpret_cast<unsigned char *>(p + i);
    for (int a = 0, b = 7; a < b; a++, b--) std::swap(c[a], c[b]);
  }
}

// Text of a header line before its label (the value field), trimmed.
std::string value_of(const char *line) {
  std::string s(line);
  while (!s.empty() && (s.back() == '\n' || s.back() == '\r')) s.pop_back();
  return s;
}

void copy_str(char *dst, size_t cap, const std::string &s) {
  const size_t n = std::min(cap - 1, s.size());
  std::memcpy(dst, s.data(), n);
  dst[n] = '\0';
}

}  // namespace

extern "C" int sx_field_write(const char *path, const sx_field_header *h, const double *const *fields,
                              int plane_stride) {
  if (!path || !h || !fields || h->np < 1 || h->nz < 1 || h->nel < 1) return SX_ERR_ARG;
  const int nfields = (int)std::strlen(h->fields);
  const size_t nP = (size_t)h->nel * h->np * h->np;
  if (nfields < 1 || plane_stride < (long long)nP) return SX_ERR_ARG;
  FILE *fp = std::fopen(path, "wb");
  if (!fp) {
    set_error("sx_field_write: cannot open %s", path);
    return SX_ERR_ARG;
  }
  char created[64];
  const time_t tp = time(nullptr);
  std::strftime(created, sizeof(created), "%a %b %d %H:%M:%S %Y", std::localtime(&tp));
  char fmt[64];
  std::snprintf(fmt, sizeof(fmt), "binary IEEE %s-endian", host_little_endian() ? "little" : "big");
  int ok = 1;
  ok &= std::fprintf(fp, "%-25s Session\n", h->session) > 0;
  ok &= std::fprintf(fp, "%-25s Created\n", created) > 0;
  ok &= std::fprintf(fp, "%-5d %-5d %-5d %-5d   Nr, Ns, Nz, Elements\n", h->np, h->np, h->nz, h->nel) > 0;
  ok &= std::fprintf(fp, "%-25d Step\n", h->step) > 0;
  ok &= std::fprintf(fp, "%-25.6g Time\n", h->time) > 0;
  ok &= std::fprintf(fp, "%-25.6g Time step\n", h->dt) > 0;
  ok &= std::fprintf(fp, "%-25.6g Kinvis\n", h->kinvis) > 0;
  ok &= std::fprintf(fp, "%-25.6g Beta\n", h->beta) > 0;
  ok &= std::fprintf(fp, "%-25s Fields written\n", h->fields) > 0;
  ok &= std::fprintf(fp, "%-25s Format\n", fmt) > 0;
  for (int f = 0; f < nfields && ok; f++)
    for (int z = 0; z < h->nz && ok; z++)
      ok &= std::fwrite(fields[f] + (size_t)z * plane_stride, sizeof(double), nP, fp) == nP;
  ok &= std::fclose(fp) == 0;
  if (!ok) {
    set_error("sx_field_write: failed writing %s", path);
    return SX_ERR_ARG;
  }
  return SX_OK;
}

extern "C" int sx_field_read_header(const char *path, sx_field_header *h) {
  if (!path || !h) return SX_ERR_ARG;
  FILE *fp = std::fopen(path, "rb");
  if (!fp) {
    set_error("sx_field_read_header: cannot open %s", path);
    return SX_ERR_ARG;
  }
  std::memset(h, 0, sizeof(*h));
  char line[10][512];
  int n = 0;
  for (; n < 10; n++)
    if (!std::fgets(line[n], sizeof(line[n]), fp)) break;
  std::fclose(fp);
  if (n < 10 || !std::strstr(line[0], "Session")) {
    set_error("sx_field_read_header: %s is not a field file", path);
    return SX_ERR_ARG;
  }
  int nr = 0, ns = 0;
  if (std::sscanf(line[2], "%d %d %d %d", &nr, &ns, &h->nz, &h->nel) != 4 || nr != ns || nr < 1 || h->nz < 1 ||
      h->nel < 1) {
    set_error("sx_field_read_header: bad size line in %s", path);
    return SX_ERR_ARG;
  }
  h->np = nr;
  std::string sess = value_of(line[0]);
  sess = sess.substr(0, sess.rfind("Session"));
  while (!sess.empty() && sess.back() == ' ') sess.pop_back();
  copy_str(h->session, sizeof(h->session), sess);
  std::sscanf(line[3], "%d", &h->step);
  std::sscanf(line[4], "%lf", &h->time);
  std::sscanf(line[5], "%lf", &h->dt);
  std::sscanf(line[6], "%lf", &h->kinvis);
  std::sscanf(line[7], "%lf", &h->beta);
  int k = 0;  // the field names: the leading alphanumeric run (compare.cpp:163-167)
  while (k < (int)sizeof(h->fields) - 1 && std::isalnum((unsigned char)line[8][k])) {
    h->fields[k] = line[8][k];
    k++;
  }
  h->fields[k] = '\0';
  if (!std::strstr(line[9], "binary")) {
    set_error("sx_field_read_header: %s is not in binary format", path);
    return SX_ERR_UNSUPPORTED;
  }
  const bool big = std::strstr(line[9], "big") != nullptr, little = std::strstr(line[9], "little") != nullptr;
  h->swapped = ((big && host_little_endian()) || (little && !host_little_endian())) ? 1 : 0;
  return SX_OK;
}

extern "C" int sx_field_read(const char *path, sx_field_header *h, double *const *fields, int plane_stride) {
  if (!path || !h || !fields) return SX_ERR_ARG;
  SX_TRY(sx_field_read_header(path, h));
  const int nfields = (int)std::strlen(h->fields);
  const size_t nP = (size_t)h->nel * h->np * h->np;
  if (plane_stride < (long long)nP) return SX_ERR_ARG;
  FILE *fp = std::fopen(path, "rb");
  if (!fp) return SX_ERR_ARG;
  char line[512];
  for (int n = 0; n < 10; n++)
    if (!std::fgets(line, sizeof(line), fp)) {
      std::fclose(fp);
      return SX_ERR_ARG;
    }
  int ok = 1;
  for (int f = 0; f < nfields && ok; f++) {
    if (!fields[f]) {  // a field the caller does not want: skip its planes
      ok &= std::fseek(fp, (long)(nP * sizeof(double)) * h->nz, SEEK_CUR) == 0;
      continue;
    }
    for (int z = 0; z < h->nz && ok; z++) {
      double *p = fields[f] + (size_t)z * plane_stride;
      ok &= std::fread(p, sizeof(double), nP, fp) == nP;
      if (ok && h->swapped) swap8(p, nP);
      if (ok && (size_t)plane_stride > nP) std::memset(p + nP, 0, sizeof(double) * (plane_stride - nP));
    }
  }
  std::fclose(fp);
  if (!ok) {
    set_error("sx_field_read: %s is shorter than its header says", path);
    return SX_ERR_ARG;
  }
  return SX_OK;
}

namespace {

// Per (element, plane): max |a - b| and sum (a - b)^2 Q4 over its nodes.
__global__ void k_norm_elem(const double *__restrict__ a, const double *__restrict__ b, const double *__restrict__ Q4,
                            int nel, int npnp, long long stride, double *__restrict__ emax, double *__restrict__ esq) {
  const int e = blockIdx.x, z = blockIdx.y;
  const double *pa = a + (size_t)z * stride + (size_t)e * npnp;
  const double *pb = b + (size_t)z * stride + (size_t)e * npnp;
  double mx = 0.0, sq = 0.0;
  for (int i = threadIdx.x; i < npnp; i += 32) {
    const double d = pa[i] - pb[i];
    mx = fmax(mx, fabs(d));
    sq += d * d * Q4[(size_t)e * npnp + i];
  }
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    sq += __shfl_xor_sync(0xffffffffu, sq, o);
  }
  if (threadIdx.x == 0) {
    emax[(size_t)z * nel + e] = mx;
    esq[(size_t)z * nel + e] = sq;
  }
}

// Per plane, in element order: inf = max, L2 = sum sqrt(esq) / area.
__global__ void k_norm_plane(const double *__restrict__ emax, const double *__restrict__ esq,
                             const double *__restrict__ Q4, int nel, int npnp, double *__restrict__ out) {
  const int z = blockIdx.x;
  if (threadIdx.x != 0) return;
  double mx = 0.0, l2 = 0.0, area = 0.0;
  for (int e = 0; e < nel; e++) {
    mx = fmax(mx, emax[(size_t)z * nel + e]);
    l2 += sqrt(esq[(size_t)z * nel + e]);
    double ar = 0.0;
    for (int i = 0; i < npnp; i++) ar += Q4[(size_t)e * npnp + i];
    area += ar;
  }
  out[2 * z] = mx;
  out[2 * z + 1] = l2 / area;
}

}  // namespace

extern "C" int sx_field_norms(sx_mesh mesh, const double *d_computed, const double *d_exact, int nz,
                              int plane_stride, double *norms, void *stream) {
  if (!mesh || !d_computed || !d_exact || !norms || nz < 1 || plane_stride < mesh->nel * mesh->npnp)
    return SX_ERR_ARG;
  SX_TRY(check_mesh_device(*mesh, "sx_field_norms"));
  cudaStream_t st = (cudaStream_t)stream;
  DBuf<double> emax, esq, out;
  SX_TRY(emax.alloc_on((size_t)nz * mesh->nel, st));
  SX_TRY(esq.alloc_on((size_t)nz * mesh->nel, st));
  SX_TRY(out.alloc_on((size_t)2 * nz, st));
  k_norm_elem<<<dim3(mesh->nel, nz), 32, 0, st>>>(d_exact, d_computed, mesh->dQ4.p, mesh->nel, mesh->npnp,
                                                   plane_stride, emax.p, esq.p);
  k_norm_plane<<<nz, 32, 0, st>>>(emax.p, esq.p, mesh->dQ4.p, mesh->nel, mesh->npnp, out.p);
  SX_CUDA(cudaGetLastError());
  SX_CUDA(cudaMemcpyAsync(norms, out.p, sizeof(double) * 2 * nz, cudaMemcpyDeviceToHost, st));
  SX_CUDA(cudaStreamSynchronize(st));
  return SX_OK;
}

// ---------------------------------------------------------------------------
// Numbering files (session.num)
// ---------------------------------------------------------------------------

namespace {

// The next whitespace-separated word of a text stream; empty at the end.
struct Words {
  FILE *fp;
  std::string next() {
    std::string w;
    int c;
    while ((c = std::fgetc(fp)) != EOF && std::isspace(c)) {
    }
    while (c != EOF && !std::isspace(c)) {
      w.push_back((char)c);
      c = std::fgetc(fp);
    }
    if (c != EOF) std::ungetc(c, fp);  // the word's end stays, as after `stream >> word`
    return w;
  }
  void rest_of_line() {
    int c;
    while ((c = std::fgetc(fp)) != EOF && c != '\n') {
    }
  }
  bool integer(long long &v) {
    const std::string w = next();
    char *end = nullptr;
    v = std::strtoll(w.c_str(), &end, 10);
    return !w.empty() && end && *end == '\0';
  }
};

}  // namespace

extern "C" int sx_numbering_read(const char *path, char field, int nel, int np, int *btog, int *bmask, int *nglobal,
                                 int *nsolve, int *nband, char *set_fields, int set_fields_cap) {
  if (!path || nel < 1 || np < 2 || !btog || !bmask) return SX_ERR_ARG;
  FILE *fp = std::fopen(path, "r");
  if (!fp) {
    set_error("sx_numbering_read: cannot open %s", path);
    return SX_ERR_ARG;
  }
  Words in{fp};
  auto fail = [&](const char *what, const std::string &got) {
    set_error("sx_numbering_read: %s: expected %s, found \"%s\"", path, what, got.c_str());
    std::fclose(fp);
    return SX_ERR_ARG;
  };
  // "# FIELDS : uvp", then the rule line (BCmgr::buildnum, src/bcmgr.cpp:640-660)
  std::string w;
  if ((w = in.next()) != "#") return fail("#", w);
  if ((w = in.next()) != "FIELDS") return fail("FIELDS", w);
  in.next();
  const std::string fields = in.next();
  in.rest_of_line();
  in.rest_of_line();
  long long nset = 0;
  if ((w = in.next()) != "#") return fail("#", w);
  if (!in.integer(nset) || nset < 1 || nset > 16) return fail("a count of number sets", "?");
  in.next();  // NUMBER
  in.next();  // SETS
  in.next();  // :
  std::vector<std::string> sets((size_t)nset);
  int which = -1;
  for (int i = 0; i < nset; i++) {
    sets[i] = in.next();
    if (which < 0 && sets[i].find(field) != std::string::npos) which = i;
  }
  if (which < 0) {
    set_error("sx_numbering_read: %s has no number set for field '%c' (fields \"%s\")", path, field, fields.c_str());
    std::fclose(fp);
    return SX_ERR_ARG;
  }
  const int next = 4 * (np - 1), ntot = nel * next;
  // the per-set summary lines, in the order enumerate writes them
  // (utility/enumerate.cpp:426-513); the reader's consistency checks
  const char *keys[] = {"NEL", "NP_MAX", "NEXT_MAX", "NINT_MAX", "NTOTAL", "NBOUNDARY", "NGLOBAL", "NSOLVE",
                        "OPTIMIZATION", "BANDWIDTH"};
  long long vals[10][16];
  for (int k = 0; k < 10; k++) {
    if ((w = in.next()) != "#") return fail("#", w);
    if ((w = in.next()) != keys[k]) return fail(keys[k], w);
    in.next();  // :
    for (int i = 0; i < nset; i++)
      if (!in.integer(vals[k][i])) return fail("an integer", keys[k]);
  }
  auto val = [&](int k) { return vals[k][which]; };
  if (val(0) != nel) {
    set_error("sx_numbering_read: mismatch in number of elements: %lld vs. %d", val(0), nel);
    std::fclose(fp);
    return SX_ERR_ARG;
  }
  if (val(1) != np) {
    set_error("sx_numbering_read: mismatch in element order: %lld vs. %d", val(1), np);
    std::fclose(fp);
    return SX_ERR_ARG;
  }
  if (val(5) != ntot) {
    set_error("sx_numbering_read: mismatch in number of boundary nodes: %lld vs. %d", val(5), ntot);
    std::fclose(fp);
    return SX_ERR_ARG;
  }
  in.rest_of_line();
  in.rest_of_line();  // rule
  in.rest_of_line();  // column titles
  for (int i = 0; i < ntot; i++) {
    long long e, s, o;
    if (!in.integer(e) || !in.integer(s) || !in.integer(o)) return fail("element, side, offset", "?");
    for (int j = 0; j < nset; j++) {
      long long g, m;
      if (!in.integer(g) || !in.integer(m)) return fail("bmap and mask", "?");
      if (j == which) {
        if (g < 0 || g >= val(6) || (m != 0 && m != 1)) {
          set_error("sx_numbering_read: %s: node %d: global number %lld / mask %lld out of range", path, i, g, m);
          std::fclose(fp);
          return SX_ERR_ARG;
        }
        btog[i] = (int)g;
        bmask[i] = (int)m;
      }
    }
  }
  std::fclose(fp);
  if (nglobal) *nglobal = (int)val(6);
  if (nsolve) *nsolve = (int)val(7);
  if (nband) *nband = (int)val(9);
  if (set_fields && set_fields_cap > 0) copy_str(set_fields, (size_t)set_fields_cap, sets[which]);
  return SX_OK;
}

extern "C" int sx_numbering_write(const char *path, const char *fields, int nset, const char *const *set_fields,
                                  int nel, int np, const int *const *btog, const int *const *bmask,
                                  const int *nglobal, const int *nsolve, const int *nband, int optimization) {
  if (!path || !fields || nset < 1 || nset > 16 || !set_fields || nel < 1 || np < 2 || !btog || !bmask ||
      !nglobal || !nsolve || !nband)
    return SX_ERR_ARG;
  FILE *fp = std::fopen(path, "w");
  if (!fp) {
    set_error("sx_numbering_write: cannot open %s", path);
    return SX_ERR_ARG;
  }
  const int next = 4 * (np - 1), nint = (np - 2) * (np - 2);
  std::fprintf(fp, "# FIELDS         :  %s\n", fields);
  std::fprintf(fp, "# ----------------");
  for (int j = 0; j < nset; j++) std::fprintf(fp, "  -------------");
  std::fprintf(fp, "\n# %d NUMBER SETS  :", nset);
  for (int j = 0; j < nset; j++) std::fprintf(fp, "%15s", set_fields[j]);
  const long long row[10] = {nel, np, next, nint, (long long)nel * np * np, (long long)nel * next, 0, 0,
                             optimization, 0};
  const char *keys[] = {"NEL           ", "NP_MAX        ", "NEXT_MAX      ", "NINT_MAX      ",
                        "NTOTAL        ", "NBOUNDARY     ", "NGLOBAL       ", "NSOLVE        ",
                        "OPTIMIZATION  ", "BANDWIDTH     "};
  for (int k = 0; k < 10; k++) {
    std::fprintf(fp, "\n# %s :", keys[k]);
    for (int j = 0; j < nset; j++)
      std::fprintf(fp, "%15lld", k == 6 ? (long long)nglobal[j] : k == 7 ? (long long)nsolve[j]
                                                           : k == 9 ? (long long)nband[j] : row[k]);
  }
  std::fprintf(fp, "\n# ----------------");
  for (int j = 0; j < nset; j++) std::fprintf(fp, "  -------------");
  std::fprintf(fp, "\n# elmt  side offst");
  for (int j = 0; j < nset; j++) std::fprintf(fp, "     bmap  mask");
  std::fprintf(fp, "\n");
  const int nedge = np - 1;
  for (int i = 0, k = 1; k <= nel; k++)
    for (int side = 1; side <= 4; side++)
      for (int soff = 0; soff < nedge; soff++, i++) {
        std::fprintf(fp, "%6d%6d%6d", k, side, soff);
        for (int j = 0; j < nset; j++) std::fprintf(fp, "%9d%6d", btog[j][i], bmask[j][i]);
        std::fprintf(fp, "\n");
      }
  const int ok = std::ferror(fp) == 0;
  std::fclose(fp);
  if (!ok) {
    set_error("sx_numbering_write: failed writing %s", path);
    return SX_ERR_ARG;
  }
  return SX_OK;
}
