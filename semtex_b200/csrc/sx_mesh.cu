// sx_mesh.cu -- host-side element geometry and numbering tables, kept
// resident on the device.
//
// Reference: Element::Element / Element::mapping (src/element.cpp:30-100,
// 1281-1436), Element::sideGeom (src/element.cpp:1653-1780), femlib
// quadrature (femlib/polylib.c:312-352, 513-560) and edge maps
// (femlib/mapping.c:46-132), emask (src/bcmgr.cpp:797-803).
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <algorithm>
#include <map>
#include <mutex>
#include <numeric>

#include "sx_internal.h"

namespace sx {

static thread_local char g_err[512];

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

const char *last_error() { return g_err; }

// GLL points z (roots of (1-z^2) P'_N), weights 2/(N(N+1) P_N(z)^2) and the
// Lagrange derivative matrix D[i][j] = h_j'(z_i), from the closed forms for
// Legendre-Lobatto nodes.  Interior roots by Newton iteration in long double.
static void legendre(int n, long double x, long double &p, long double &dp) {
  long double p0 = 1.0L, p1 = x, d0 = 0.0L, d1 = 1.0L;
  if (n == 0) {
    p = 1.0L;
    dp = 0.0L;
    return;
  }
  for (int k = 2; k <= n; k++) {
    long double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
    long double d2 = d0 + (2 * k - 1) * p1;
    p0 = p1;
    p1 = p2;
    d0 = d1;
    d1 = d2;
  }
  p = p1;
  dp = d1;
}

void gll_tables(int np, std::vector<double> &z, std::vector<double> &w, std::vector<double> &D) {
  const int N = np - 1;
  std::vector<long double> zl(np), pn(np);
  zl[0] = -1.0L;
  zl[N] = 1.0L;
  const long double pi = 3.14159265358979323846264338327950288L;
  for (int i = 1; i < N; i++) {
    long double x = -cosl(pi * i / N);
    for (int it = 0; it < 100; it++) {
      long double p, dp;
      legendre(N, x, p, dp);
      long double d2 = (2.0L * x * dp - N * (N + 1.0L) * p) / (1.0L - x * x);
      long double dx = dp / d2;
      x -= dx;
      if (fabsl(dx) < 1e-30L) break;
    }
    zl[i] = x;
  }
  for (int i = 0; i < np / 2; i++) {
    long double a = 0.5L * (zl[N - i] - zl[i]);
    zl[i] = -a;
    zl[N - i] = a;
  }
  if (np % 2) zl[N / 2] = 0.0L;
  z.assign(np, 0.0);
  w.assign(np, 0.0);
  D.assign(np * np, 0.0);
  for (int i = 0; i < np; i++) {
    long double dp;
    legendre(N, zl[i], pn[i], dp);
    z[i] = (double)zl[i];
    w[i] = (double)(2.0L / (N * (N + 1.0L) * pn[i] * pn[i]));
  }
  for (int i = 0; i < np; i++)
    for (int j = 0; j < np; j++) {
      long double d;
      if (i != j)
        d = pn[i] / (pn[j] * (zl[i] - zl[j]));
      else if (i == 0)
        d = -N * (N + 1.0L) / 4.0L;
      else if (i == N)
        d = N * (N + 1.0L) / 4.0L;
      else
        d = 0.0L;
      D[i * np + j] = (double)d;
    }
}

// Edge-major CCW permutation and its inverse.
void edge_maps(int np, std::vector<int> &emap, std::vector<int> &pmap) {
  emap.assign(np * np, 0);
  pmap.assign(np * np, 0);
  int k = 0, n = 0;
  const int steps[4] = {1, np, -1, -np};
  for (int s = 0; s < 4; s++)
    for (int i = 1; i < np; i++) {
      emap[k++] = n;
      n += steps[s];
    }
  for (int i = 1; i < np - 1; i++)
    for (int j = 1; j < np - 1; j++) emap[k++] = i * np + j;
  for (int i = 0; i < np * np; i++) pmap[emap[i]] = i;
}

static void mxm(const double *A, int m, const double *B, int k, double *C, int n) {
  for (int i = 0; i < m; i++)
    for (int j = 0; j < n; j++) {
      double s = 0.0;
      for (int p = 0; p < k; p++) s += A[i * k + p] * B[p * n + j];
      C[i * n + j] = s;
    }
}

static double nrm2(int n, const double *a) {
  double s = 0.0;
  for (int i = 0; i < n; i++) s += a[i] * a[i];
  return std::sqrt(s);
}

// Geometric factors of one element (Cartesian, GLL): Q1..Q4 carry the
// quadrature weights, Q8 = Q4 is the mass (src/element.cpp:1340-1436).
static int element_geometry(sx_mesh_s &M, int e, const double *x, const double *y) {
  const int np = M.np, nn = M.npnp;
  std::vector<double> DT(nn), dxdr(nn), dxds(nn), dydr(nn), dyds(nn);
  for (int i = 0; i < np; i++)
    for (int j = 0; j < np; j++) DT[j * np + i] = M.D[i * np + j];
  mxm(x, np, DT.data(), np, dxdr.data(), np);
  mxm(M.D.data(), np, x, np, dxds.data(), np);
  mxm(y, np, DT.data(), np, dydr.data(), np);
  mxm(M.D.data(), np, y, np, dyds.data(), np);
  double *Q1 = &M.Q1[(size_t)e * nn], *Q2 = &M.Q2[(size_t)e * nn], *Q3 = &M.Q3[(size_t)e * nn];
  double *Q4 = &M.Q4[(size_t)e * nn], *Q8 = &M.Q8[(size_t)e * nn];
  const double EPS = 4 * EPSDP;
  for (int i = 0; i < np; i++)
    for (int j = 0; j < np; j++) {
      const int k = i * np + j;
      const double jac = dxdr[k] * dyds[k] - dxds[k] * dydr[k];
      if (jac < EPS) {
        set_error("Jacobian of element %d nonpositive", e + 1);
        return SX_ERR_JACOBIAN;
      }
      const double ww = M.w[i] * M.w[j];
      Q1[k] = (dxds[k] * dxds[k] + dyds[k] * dyds[k]) / jac * ww;
      Q2[k] = (dxdr[k] * dxdr[k] + dydr[k] * dydr[k]) / jac * ww;
      Q3[k] = (-(dydr[k] * dyds[k]) - dxdr[k] * dxds[k]) / jac * ww;
      Q4[k] = jac * ww;
      Q8[k] = Q4[k];
    }
  // Null-mapping: drop Q3 for undistorted elements (src/element.cpp:1431-1435).
  M.hasQ3[e] = nrm2(nn, Q3) >= EPS;
  if (!M.hasQ3[e]) std::memset(Q3, 0, sizeof(double) * nn);
  // Inverse mapping partials (src/element.cpp:1403-1411), each dropped by
  // the same null-mapping test (:1431-1434); a dropped partial reads as 0.
  if (M.drdx.empty()) return SX_OK;  // geometry-only callers
  double *rx = &M.drdx[(size_t)e * nn], *ry = &M.drdy[(size_t)e * nn];
  double *sx_ = &M.dsdx[(size_t)e * nn], *sy = &M.dsdy[(size_t)e * nn];
  for (int k = 0; k < nn; k++) {
    const double jac = dxdr[k] * dyds[k] - dxds[k] * dydr[k];
    rx[k] = dyds[k] / jac;
    ry[k] = -dxds[k] / jac;
    sx_[k] = -dydr[k] / jac;
    sy[k] = dxdr[k] / jac;
  }
  for (double *a : {rx, ry, sx_, sy})
    if (nrm2(nn, a) < EPS) std::memset(a, 0, sizeof(double) * nn);
  return SX_OK;
}

// Edge "area" factor |d(x,y)/dr| w at the side nodes, in the order the
// reference stores it (src/element.cpp:1679-1780).
static void side_area(const sx_mesh_s &M, const double *x, const double *y, int side, double *area) {
  const int np = M.np;
  int low, skip;
  switch (side) {
    case 0: low = 0; skip = 1; break;
    case 1: low = np - 1; skip = np; break;
    case 2: low = np * (np - 1); skip = 1; break;
    default: low = 0; skip = np; break;
  }
  for (int i = 0; i < np; i++) {
    double xr = 0.0, yr = 0.0;
    for (int k = 0; k < np; k++) {
      xr += M.D[i * np + k] * x[low + k * skip];
      yr += M.D[i * np + k] * y[low + k * skip];
    }
    area[i] = std::sqrt(xr * xr + yr * yr) * M.w[i];
  }
}

}  // namespace sx

sx::MeshView sx_mesh_s::view() const {
  sx::MeshView v;
  v.np = np; v.npnp = npnp; v.next = next; v.nint = nint; v.nel = nel;
  v.nglobal = nglobal; v.nsolve_ns = nsolve; v.nband = nband;
  v.D = dD.p; v.emap = demap.p;
  v.Q1 = dQ1.p; v.Q2 = dQ2.p; v.Q3 = dQ3.p; v.Q4 = dQ4.p; v.Q8 = dQ8.p;
  v.Q1f = dQ1f.p; v.Q2f = dQ2f.p; v.Q3f = dQ3f.p; v.Q4f = dQ4f.p; v.Df = dDf.p;
  v.hasQ3 = dhasQ3.p;
  v.btog = dbtog.p; v.bmask = dbmask.p; v.emask = demask.p;
  v.g2e_ptr = dg2e_ptr.p; v.g2e_idx = dg2e_idx.p; v.g2e_last = dg2e_last.p;
  v.g2e4 = dg2e4.p; v.owner = downer.p;
  v.e2w4 = de2w4.p; v.Gf = dGf.p; v.pmap = dpmap.p;
  v.nbound = nbound; v.b_elmt = dbe.p; v.b_side = dbs.p; v.b_kind = dbk.p;
  v.b_K = dK.p; v.b_C = dC.p; v.b_area = darea.p;
  v.nat_ptr = dnat_ptr.p; v.nat_idx = dnat_idx.p;
  v.mixed = mixed ? 1 : 0;
  return v;
}

using namespace sx;

// Global node touched by boundary b's local line index i (Essential::set,
// src/condition.cpp:80-101).
static int bnd_node(const sx_mesh_s &M, int b, int i) {
  const int nm = M.np - 1;
  const int *bmap = &M.btog[(size_t)M.b_elmt[b] * M.next];
  const int side = M.b_side[b];
  if (i < nm) return bmap[side * nm + i];
  return side == 3 ? bmap[0] : bmap[side * nm + nm];
}

// max over nodes of diag(K)_g / diag(M)_g from the host geometry, Q3 cross
// terms left out.  The stiffness part of Element::HelmholtzDiag
// (src/element.cpp:1512-1561) at tensor node (i, j) is
//   sum_k D(k, i)^2 Q2(k, j) + sum_k Q1(i, k) D(k, j)^2
// and the mass part Q4(i, j); boundary nodes are summed over their elements.
static double stiffness_mass_ratio(const sx_mesh_s &M) {
  const int np = M.np, nn = M.npnp, next = M.next, nint = M.nint;
  std::vector<double> K((size_t)M.nglobal + (size_t)M.nel * nint, 0.0), Mm(K.size(), 0.0);
  for (int e = 0; e < M.nel; e++) {
    const double *Q1 = &M.Q1[(size_t)e * nn], *Q2 = &M.Q2[(size_t)e * nn], *Q4 = &M.Q4[(size_t)e * nn];
    for (int i = 0; i < np; i++)
      for (int j = 0; j < np; j++) {
        double k = 0.0;
        for (int m = 0; m < np; m++) {
          const double di = M.D[m * np + i], dj = M.D[m * np + j];
          k += di * di * Q2[m * np + j] + Q1[i * np + m] * dj * dj;
        }
        const int t = i * np + j, a = M.pmap[t];
        const size_t g = a < next ? (size_t)M.btog[(size_t)e * next + a]
                                  : (size_t)M.nglobal + (size_t)e * nint + (a - next);
        K[g] += k;
        Mm[g] += Q4[t];
      }
  }
  double r = 0.0;
  for (size_t g = 0; g < K.size(); g++)
    if (Mm[g] > 0.0) r = std::max(r, K[g] / Mm[g]);
  return r;
}

namespace sx {

int mesh_kratio(const sx_mesh_desc *d, double *out) {
  if (!d || !out || d->np < NP_MIN || d->np > NP_MAX || d->nel <= 0 || !d->x || !d->y || !d->btog ||
      d->nglobal <= 0)
    return SX_ERR_ARG;
  sx_mesh_s T;  // host geometry only
  const int np = d->np, nn = np * np, next = 4 * (np - 1), nel = d->nel;
  T.np = np; T.npnp = nn; T.next = next; T.nint = nn - next; T.nel = nel; T.nglobal = d->nglobal;
  gll_tables(np, T.z, T.w, T.D);
  edge_maps(np, T.emap, T.pmap);
  const size_t tot = (size_t)nel * nn, tb = (size_t)nel * next;
  T.Q1.assign(tot, 0.0); T.Q2.assign(tot, 0.0); T.Q3.assign(tot, 0.0);
  T.Q4.assign(tot, 0.0); T.Q8.assign(tot, 0.0);
  T.hasQ3.assign(nel, 0);
  for (int e = 0; e < nel; e++)
    SX_TRY(element_geometry(T, e, d->x + (size_t)e * nn, d->y + (size_t)e * nn));
  T.btog.assign(d->btog, d->btog + tb);
  for (size_t i = 0; i < tb; i++)
    if (T.btog[i] < 0 || T.btog[i] >= d->nglobal) return SX_ERR_ARG;
  *out = stiffness_mass_ratio(T);
  return SX_OK;
}

}  // namespace sx

// Device memory of meshes comes from a stream-ordered pool of their own
// (one per device), so that dropping a mesh frees its memory without the
// device-wide synchronisation of cudaFree (a server drops one per request
// while other requests run), and creating one waits for nothing but its own
// copies.  Up to MESH_POOL_KEEP bytes of freed mesh memory stay mapped for
// the next mesh.
constexpr uint64_t MESH_POOL_KEEP = uint64_t(4) << 30;

static int mesh_pool(int device, cudaMemPool_t *out) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  std::lock_guard<std::mutex> lk(mu);
  auto it = pools.find(device);
  if (it == pools.end()) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    SX_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = MESH_POOL_KEEP;
    SX_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    it = pools.emplace(device, pool).first;
  }
  *out = it->second;
  return SX_OK;
}

// The pool and a private stream for one mesh's uploads.
struct MeshUpload {
  cudaMemPool_t pool = nullptr;
  cudaStream_t s = nullptr;
  int begin(int device) {
    SX_TRY(mesh_pool(device, &pool));
    SX_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    return SX_OK;
  }
  ~MeshUpload() {
    if (s) cudaStreamDestroy(s);
  }
};

// Envelope of the condensed matrix and of its Cholesky factor, by tiles.
// Node c (< nsolve) is coupled to every solve node of the elements that hold
// it, so row c of the matrix starts at first(c) = the lowest solve node of
// those elements.  Cholesky fill stays inside this envelope (George & Liu,
// Computer Solution of Large Sparse Positive Definite Systems, 1981, ch. 4):
// U(r, c) = 0 exactly for r < first(c), in floating point too, because every
// product that forms such an entry has a zero factor.  By block columns of NB,
// column block k can be non-zero only from row block fb(k) = min first(c) / NB
// over its columns.  The tables use the suffix minimum fm(k) = min over k' >= k
// of fb(k'), a monotone hull of that staircase, so that the non-zero tiles of
// every block row are contiguous too: block column k holds jf(k) = k - fm(k)
// tiles above its diagonal, block row k the jb(k) = max{ j : fm(k + j) <= k }
// right of it.  The pressure pin (nsolve - 1) only removes a row and column,
// so the tables of nsolve hold for it as well.
// btog entries must lie in [0, nglobal) (the callers check).
static void envelope_tables(const int *btog, int nel, int next, int ns, int nband, int &nblk,
                            std::vector<int> &env) {
  const int J = (nband - 1 + NB - 1) / NB;
  nblk = (ns + NB - 1) / NB;
  std::vector<int> fm(nblk);
  for (int k = 0; k < nblk; k++) fm[k] = k;
  for (int e = 0; e < nel; e++) {
    const int *g = &btog[(size_t)e * next];
    int lo = ns;
    for (int i = 0; i < next; i++)
      if (g[i] < ns) lo = std::min(lo, g[i]);
    for (int i = 0; i < next; i++)
      if (g[i] < ns) fm[g[i] / NB] = std::min(fm[g[i] / NB], lo / NB);
  }
  for (int k = nblk - 2; k >= 0; k--) fm[k] = std::min(fm[k], fm[k + 1]);
  env.assign((size_t)2 * std::max(nblk, 1), 0);
  int c = 0;  // the last block column whose hull reaches row block k
  for (int k = 0; k < nblk; k++) {
    env[k] = std::min(J, k - fm[k]);
    c = std::max(c, k);
    while (c + 1 < nblk && fm[c + 1] <= k) c++;
    env[nblk + k] = std::min(J, c - k);
  }
}

static int band_envelope(sx_mesh_s &M) {
  envelope_tables(M.btog.data(), M.nel, M.next, M.nsolve, M.nband, M.env_nblk, M.env);
  return SX_OK;
}

extern "C" int sx_mesh_desc_envelope(const sx_mesh_desc *d, int *nblk, int *env) {
  if (!d || !nblk || d->np < 2 || d->nel <= 0 || !d->btog || d->nglobal <= 0 || d->nsolve < 0 ||
      d->nsolve > d->nglobal || d->nband <= 0) {
    set_error("invalid mesh description");
    return SX_ERR_ARG;
  }
  const int next = 4 * (d->np - 1);
  const size_t tb = (size_t)d->nel * next;
  for (size_t i = 0; i < tb; i++)
    if (d->btog[i] < 0 || d->btog[i] >= d->nglobal) {
      set_error("btog[%zu] = %d outside [0, nglobal)", i, d->btog[i]);
      return SX_ERR_ARG;
    }
  std::vector<int> tab;
  int nb = 0;
  envelope_tables(d->btog, d->nel, next, d->nsolve, d->nband, nb, tab);
  *nblk = nb;
  if (env) std::memcpy(env, tab.data(), sizeof(int) * 2 * (size_t)nb);
  return SX_OK;
}

extern "C" int sx_mesh_create(const sx_mesh_desc *d, sx_mesh *out) {
  if (!d || !out) return SX_ERR_ARG;
  *out = nullptr;
  if (d->np < NP_MIN || d->np > NP_MAX) {
    set_error("np = %d outside the supported range [%d, %d]", d->np, NP_MIN, NP_MAX);
    return SX_ERR_UNSUPPORTED;
  }
  if (d->nel <= 0 || !d->x || !d->y || !d->btog || !d->bmask || d->nglobal <= 0 ||
      d->nsolve < 0 || d->nsolve > d->nglobal || d->nband <= 0 || d->nbound < 0 ||
      (d->nbound > 0 && (!d->b_elmt || !d->b_side || !d->b_kind))) {
    set_error("invalid mesh description");
    return SX_ERR_ARG;
  }
  std::unique_ptr<sx_mesh_s> M(new sx_mesh_s());
  cudaGetDevice(&M->device);
  const int np = d->np, nn = np * np, next = 4 * (np - 1), nel = d->nel;
  M->np = np; M->npnp = nn; M->next = next; M->nint = nn - next; M->nel = nel;
  M->nglobal = d->nglobal; M->nsolve = d->nsolve; M->nband = d->nband; M->nbound = d->nbound;
  gll_tables(np, M->z, M->w, M->D);
  edge_maps(np, M->emap, M->pmap);
  const size_t tot = (size_t)nel * nn, tb = (size_t)nel * next;
  M->Q1.assign(tot, 0.0); M->Q2.assign(tot, 0.0); M->Q3.assign(tot, 0.0);
  M->Q4.assign(tot, 0.0); M->Q8.assign(tot, 0.0);
  M->drdx.assign(tot, 0.0); M->drdy.assign(tot, 0.0); M->dsdx.assign(tot, 0.0); M->dsdy.assign(tot, 0.0);
  M->hasQ3.assign(nel, 0);
  for (int e = 0; e < nel; e++)
    SX_TRY(element_geometry(*M, e, d->x + (size_t)e * nn, d->y + (size_t)e * nn));
  M->btog.assign(d->btog, d->btog + tb);
  M->bmask.assign(d->bmask, d->bmask + tb);
  for (size_t i = 0; i < tb; i++)
    if (M->btog[i] < 0 || M->btog[i] >= d->nglobal) {
      set_error("btog[%zu] = %d outside [0, nglobal)", i, M->btog[i]);
      return SX_ERR_ARG;
    }
  // Every pair of solve nodes of an element is coupled in H: their numbers
  // must lie within the declared band (the reference's assembly,
  // src/matrix.cpp:236-241, writes band_addr(m, n, nband) unchecked)
  for (int e = 0; e < nel; e++) {
    int lo = d->nglobal, hi = -1;
    for (int i = 0; i < next; i++) {
      const int g = M->btog[(size_t)e * next + i];
      if (g < d->nsolve) {
        lo = std::min(lo, g);
        hi = std::max(hi, g);
      }
    }
    if (hi >= 0 && hi - lo >= d->nband) {
      set_error("element %d couples solve nodes %d and %d, further apart than nband - 1 = %d", e, lo, hi,
                d->nband - 1);
      return SX_ERR_BAND;
    }
  }
  SX_TRY(band_envelope(*M));
  M->emask.assign(nel, 0);
  for (int e = 0; e < nel; e++)
    for (int i = 0; i < next; i++) M->emask[e] |= M->bmask[(size_t)e * next + i] != 0;
  // boundaries
  const int nb = d->nbound;
  M->b_elmt.assign(d->b_elmt, d->b_elmt + nb);
  M->b_side.assign(d->b_side, d->b_side + nb);
  M->b_kind.assign(d->b_kind, d->b_kind + nb);
  M->b_K.assign(nb, 0.0);
  M->b_C.assign(nb, 0.0);
  M->b_area.assign((size_t)std::max(nb, 1) * np, 0.0);
  for (int b = 0; b < nb; b++) {
    if (M->b_elmt[b] < 0 || M->b_elmt[b] >= nel || M->b_side[b] < 0 || M->b_side[b] > 3 ||
        M->b_kind[b] < 0 || M->b_kind[b] > 2) {
      set_error("invalid boundary %d", b);
      return SX_ERR_ARG;
    }
    if (d->b_K) M->b_K[b] = d->b_K[b];
    if (d->b_C) M->b_C[b] = d->b_C[b];
    if (M->b_kind[b] == SX_BC_MIXED) M->mixed = true;
    const size_t o = (size_t)M->b_elmt[b] * nn;
    side_area(*M, d->x + o, d->y + o, M->b_side[b], &M->b_area[(size_t)b * np]);
  }
  // Self-periodic elements (one global node twice in an element) would make
  // the per-element assembly race; the reference notes the same hazard
  // (src/element.cpp:382).  Reject them.
  for (int e = 0; e < nel; e++) {
    std::vector<int> g(&M->btog[(size_t)e * next], &M->btog[(size_t)e * next] + next);
    std::sort(g.begin(), g.end());
    if (std::adjacent_find(g.begin(), g.end()) != g.end()) {
      set_error("element %d is self-periodic (repeated global node)", e);
      return SX_ERR_UNSUPPORTED;
    }
  }
  // CSR inverse of btog in element-major order (summation order of scatr_sum).
  std::vector<int> ptr(d->nglobal + 1, 0), idx(tb), last(d->nglobal, -1);
  for (size_t i = 0; i < tb; i++) ptr[M->btog[i] + 1]++;
  for (int g = 0; g < d->nglobal; g++)
    if (ptr[g + 1] == 0) {
      set_error("global node %d is not referenced by btog (nglobal too large?)", g);
      return SX_ERR_ARG;
    }
  for (int g = 0; g < d->nglobal; g++) ptr[g + 1] += ptr[g];
  {
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    for (size_t i = 0; i < tb; i++) {
      idx[fill[M->btog[i]]++] = (int)i;
      last[M->btog[i]] = (int)i;
    }
  }
  // CSR of natural/mixed boundary terms per global node, boundary order.
  std::vector<int> nptr(d->nglobal + 1, 0), nidx;
  {
    std::vector<std::vector<int>> lists(d->nglobal);
    for (int b = 0; b < nb; b++) {
      if (M->b_kind[b] == SX_BC_ESSENTIAL) continue;
      for (int i = 0; i < np; i++) lists[bnd_node(*M, b, i)].push_back(b * np + i);
    }
    for (int g = 0; g < d->nglobal; g++) {
      nptr[g + 1] = nptr[g] + (int)lists[g].size();
      nidx.insert(nidx.end(), lists[g].begin(), lists[g].end());
    }
    if (nidx.empty()) nidx.push_back(0);
  }
  // Greedy element colouring: elements of one colour share no global node.
  {
    std::vector<int> colour(nel, -1);
    std::vector<std::vector<int>> node_elems(d->nglobal);
    for (int e = 0; e < nel; e++)
      for (int i = 0; i < next; i++) node_elems[M->btog[(size_t)e * next + i]].push_back(e);
    int ncol = 0;
    std::vector<char> used;
    for (int e = 0; e < nel; e++) {
      used.assign(ncol + 1, 0);
      for (int i = 0; i < next; i++)
        for (int o : node_elems[M->btog[(size_t)e * next + i]])
          if (colour[o] >= 0) used[colour[o]] = 1;
      int c = 0;
      while (used[c]) c++;
      colour[e] = c;
      ncol = std::max(ncol, c + 1);
    }
    M->colour_ptr.assign(ncol + 1, 0);
    for (int e = 0; e < nel; e++) M->colour_ptr[colour[e] + 1]++;
    for (int c = 0; c < ncol; c++) M->colour_ptr[c + 1] += M->colour_ptr[c];
    M->colour_elmt.assign(nel, 0);
    std::vector<int> fill(M->colour_ptr.begin(), M->colour_ptr.end() - 1);
    for (int e = 0; e < nel; e++) M->colour_elmt[fill[colour[e]]++] = e;
  }
  // Inverse of the assembled boundary mass: unity summed into the global
  // numbering with the Q4 weights, element after element (bndryDsSum,
  // src/element.cpp:464-487, as BCmgr::buildnum uses it, src/bcmgr.cpp:805-821).
  M->imass.assign(d->nglobal, 0.0);
  for (int e = 0; e < nel; e++)
    for (int i = 0; i < next; i++)
      M->imass[M->btog[(size_t)e * next + i]] += M->Q4[(size_t)e * nn + M->emap[i]];
  for (int g = 0; g < d->nglobal; g++) M->imass[g] = 1.0 / M->imass[g];
  // FP32 copies of the geometry for the mixed-precision operator.
  std::vector<float> f1(tot), f2(tot), f3(tot), f4(tot);
  for (size_t i = 0; i < tot; i++) {
    f1[i] = (float)M->Q1[i]; f2[i] = (float)M->Q2[i];
    f3[i] = (float)M->Q3[i]; f4[i] = (float)M->Q4[i];
  }
  MeshUpload up;
  SX_TRY(up.begin(M->device));
  SX_TRY(M->dD.upload_in(M->D.data(), nn, up.pool, up.s));
  SX_TRY(M->demap.upload_in(M->emap.data(), nn, up.pool, up.s));
  SX_TRY(M->dQ1.upload_in(M->Q1.data(), tot, up.pool, up.s));
  SX_TRY(M->dQ2.upload_in(M->Q2.data(), tot, up.pool, up.s));
  SX_TRY(M->dQ3.upload_in(M->Q3.data(), tot, up.pool, up.s));
  SX_TRY(M->dQ4.upload_in(M->Q4.data(), tot, up.pool, up.s));
  SX_TRY(M->dQ8.upload_in(M->Q8.data(), tot, up.pool, up.s));
  SX_TRY(M->ddrdx.upload_in(M->drdx.data(), tot, up.pool, up.s));
  SX_TRY(M->ddrdy.upload_in(M->drdy.data(), tot, up.pool, up.s));
  SX_TRY(M->ddsdx.upload_in(M->dsdx.data(), tot, up.pool, up.s));
  SX_TRY(M->ddsdy.upload_in(M->dsdy.data(), tot, up.pool, up.s));
  SX_TRY(M->dimass.upload_in(M->imass.data(), M->imass.size(), up.pool, up.s));
  SX_TRY(M->dQ1f.upload_in(f1.data(), tot, up.pool, up.s));
  SX_TRY(M->dQ2f.upload_in(f2.data(), tot, up.pool, up.s));
  SX_TRY(M->dQ3f.upload_in(f3.data(), tot, up.pool, up.s));
  SX_TRY(M->dQ4f.upload_in(f4.data(), tot, up.pool, up.s));
  {
    std::vector<float4> gf(tot);
    for (size_t i = 0; i < tot; i++) gf[i] = make_float4(f1[i], f2[i], f3[i], f4[i]);
    SX_TRY(M->dGf.upload_in(gf.data(), tot, up.pool, up.s));
  }
  SX_TRY(M->dpmap.upload_in(M->pmap.data(), nn, up.pool, up.s));
  M->kratio = stiffness_mass_ratio(*M);
  std::vector<float> df(M->D.begin(), M->D.end());
  SX_TRY(M->dDf.upload_in(df.data(), df.size(), up.pool, up.s));
  SX_TRY(M->dhasQ3.upload_in(M->hasQ3.data(), nel, up.pool, up.s));
  SX_TRY(M->dbtog.upload_in(M->btog.data(), tb, up.pool, up.s));
  SX_TRY(M->denv.upload_in(M->env.data(), M->env.size(), up.pool, up.s));
  SX_TRY(M->dbmask.upload_in(M->bmask.data(), tb, up.pool, up.s));
  SX_TRY(M->demask.upload_in(M->emask.data(), nel, up.pool, up.s));
  SX_TRY(M->dg2e_ptr.upload_in(ptr.data(), ptr.size(), up.pool, up.s));
  SX_TRY(M->dg2e_idx.upload_in(idx.data(), idx.size(), up.pool, up.s));
  SX_TRY(M->dg2e_last.upload_in(last.data(), last.size(), up.pool, up.s));
  {
    std::vector<int4> g4(d->nglobal);
    for (int g = 0; g < d->nglobal; g++) {
      int v[4] = {-1, -1, -1, -1};
      const int n = ptr[g + 1] - ptr[g];
      for (int k = 0; k < std::min(n, 4); k++) v[k] = idx[ptr[g] + k];
      if (n > 4) v[3] = -2;  // more than 4 contributions: walk the CSR
      g4[g] = make_int4(v[0], v[1], v[2], v[3]);
    }
    SX_TRY(M->dg2e4.upload_in(g4.data(), g4.size(), up.pool, up.s));
    // per element slot: the holders of its node as (element << 8 | tensor
    // node), the element-layout address of their A u (nel < 2^23, np^2 < 256)
    if (nel >= (1 << 23)) {
      set_error("%d elements: the element-layout gather tables hold at most 2^23", nel);
      return SX_ERR_UNSUPPORTED;
    }
    auto pack = [&](int ei) { return ei < 0 ? ei : ((ei / next) << 8) | M->emap[ei % next]; };
    std::vector<int4> e4((size_t)nel * next);
    for (size_t k = 0; k < e4.size(); k++) {
      const int4 q = g4[M->btog[k]];
      e4[k] = make_int4(pack(q.x), pack(q.y), pack(q.z), q.w == -2 ? -2 : pack(q.w));
    }
    SX_TRY(M->de2w4.upload_in(e4.data(), e4.size(), up.pool, up.s));
    std::vector<unsigned long long> own(nel, 0ull);
    for (int e = 0; e < nel; e++)
      for (int a = 0; a < next; a++)
        if (last[M->btog[(size_t)e * next + a]] == e * next + a) own[e] |= 1ull << a;
    SX_TRY(M->downer.upload_in(own.data(), own.size(), up.pool, up.s));
  }
  std::vector<int> be(M->b_elmt), bs(M->b_side), bk(M->b_kind);
  if (nb == 0) { be.push_back(0); bs.push_back(0); bk.push_back(0); M->b_K.push_back(0); M->b_C.push_back(0); }
  SX_TRY(M->dbe.upload_in(be.data(), be.size(), up.pool, up.s));
  SX_TRY(M->dbs.upload_in(bs.data(), bs.size(), up.pool, up.s));
  SX_TRY(M->dbk.upload_in(bk.data(), bk.size(), up.pool, up.s));
  SX_TRY(M->dK.upload_in(M->b_K.data(), M->b_K.size(), up.pool, up.s));
  SX_TRY(M->dC.upload_in(M->b_C.data(), M->b_C.size(), up.pool, up.s));
  SX_TRY(M->darea.upload_in(M->b_area.data(), M->b_area.size(), up.pool, up.s));
  SX_TRY(M->dnat_ptr.upload_in(nptr.data(), nptr.size(), up.pool, up.s));
  SX_TRY(M->dnat_idx.upload_in(nidx.data(), nidx.size(), up.pool, up.s));
  SX_TRY(M->dcolour_elmt.upload_in(M->colour_elmt.data(), M->colour_elmt.size(), up.pool, up.s));
  *out = M.release();
  return SX_OK;
}

extern "C" int sx_mesh_destroy(sx_mesh m) {
  // the mesh's memory is freed stream-ordered: work the caller enqueued with
  // it (on any stream) must finish first
  if (m) {
    int dev = -1;
    cudaGetDevice(&dev);
    cudaSetDevice(m->device);
    cudaDeviceSynchronize();
    cudaSetDevice(dev);
  }
  delete m;
  return SX_OK;
}

extern "C" int sx_mesh_geometry(sx_mesh m, int e, double *q1, double *q2, double *q3, double *q4,
                                double *q8) {
  if (!m || e < 0 || e >= m->nel) return SX_ERR_ARG;
  const size_t o = (size_t)e * m->npnp, n = m->npnp;
  if (q1) std::memcpy(q1, &m->Q1[o], n * 8);
  if (q2) std::memcpy(q2, &m->Q2[o], n * 8);
  if (q3) std::memcpy(q3, &m->Q3[o], n * 8);
  if (q4) std::memcpy(q4, &m->Q4[o], n * 8);
  if (q8) std::memcpy(q8, &m->Q8[o], n * 8);
  return SX_OK;
}

extern "C" int sx_mesh_envelope(sx_mesh m, int *nblk, int *env) {
  if (!m || !nblk) return SX_ERR_ARG;
  *nblk = m->env_nblk;
  if (env) std::memcpy(env, m->env.data(), sizeof(int) * 2 * (size_t)m->env_nblk);
  return SX_OK;
}

extern "C" int sx_mesh_partials(sx_mesh m, int e, double *drdx, double *drdy, double *dsdx, double *dsdy,
                                double *imass) {
  if (!m || e < 0 || e >= m->nel) return SX_ERR_ARG;
  const size_t o = (size_t)e * m->npnp, n = m->npnp;
  if (drdx) std::memcpy(drdx, &m->drdx[o], n * 8);
  if (drdy) std::memcpy(drdy, &m->drdy[o], n * 8);
  if (dsdx) std::memcpy(dsdx, &m->dsdx[o], n * 8);
  if (dsdy) std::memcpy(dsdy, &m->dsdy[o], n * 8);
  if (imass) std::memcpy(imass, m->imass.data(), m->imass.size() * 8);
  return SX_OK;
}
