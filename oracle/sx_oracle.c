/*
 * sx_oracle.c -- CPU ORACLE for the per-Fourier-mode Helmholtz solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain-C restatement of the
 * reference (semtex) algorithm for the elliptic solve behind
 * Field::solve / ModalMatrixSys / MatrixSys / Element.  It is used by the
 * test-suite, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg
 * as the CHECKER; the product (semtex_b200/) never links, imports or calls
 * it.
 *
 * Parity pins: GLL tables are checked against the reference's own
 * femlib/polylib.c compiled into oracle/_ref (when the reference tree is
 * present), and whole solves are checked against the reference's regression
 * goldens regress/{helmholtz1,poisson1,laplace1,laplace4,mixed1,laplace3}.ok
 * (discretisation error vs the analytic solution, printed by
 * utility/compare.cpp:229-235 to 3 significant digits).
 *
 * The BLAS/LAPACK kernels the reference calls (dgetrf/dgetri, dpbtrf,
 * dpbtrs, dgemv, dgemm) come from an external, unpinned LAPACK
 * (CMakeLists.txt:42-43).  They are restated here from LAPACK's published
 * unblocked algorithms (dgetf2/dgetri, dpbtf2, dtbsv); results agree with
 * any LAPACK to rounding.
 *
 * Conventions (reference file:line):
 *   - equation: div grad u - lambda^2 u = f            (src/field.h:15-21)
 *   - element storage: np*np row-major per element      (src/element.h:23-24)
 *   - emap/pmap edge-major permutation                  (femlib/mapping.c:46-132)
 *   - hbb/hbi/hii row-major, band in LAPACK "U" storage (src/matrix.cpp:221-241,
 *                                                        veclib/lapack.h:107-108)
 */

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define EPSDP 6.0e-14 /* veclib/utility.h:39 */
#define EPSSP 6.0e-7  /* veclib/utility.h:35 */

/* ------------------------------------------------------------------------ */
/* Gauss-Lobatto-Legendre points, weights, derivative matrix.               */
/* Restates femlib/polylib.c:312-352 (zwglj, alpha=beta=0) and              */
/* femlib/polylib.c:513-560 (Dglj): z = roots of (1-z^2) P'_N(z), weights   */
/* w_i = 2/(N(N+1) P_N(z_i)^2), D[i][j] = h_j'(z_i) with the closed forms   */
/* P_N(z_i)/(P_N(z_j)(z_i-z_j)), -N(N+1)/4, +N(N+1)/4, 0 on the diagonal.   */
/* The interior roots are found by Newton iteration in long double.         */
/* ------------------------------------------------------------------------ */

static void legendre_ld(int n, long double x, long double *p, long double *dp)
{
  long double p0 = 1.0L, p1 = x, d0 = 0.0L, d1 = 1.0L;
  if (n == 0) { *p = 1.0L; *dp = 0.0L; return; }
  for (int k = 2; k <= n; k++) {
    long double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
    long double d2 = d0 + (2 * k - 1) * p1;
    p0 = p1; p1 = p2; d0 = d1; d1 = d2;
  }
  *p = p1; *dp = d1;
}

int orc_gll(int np, double *z, double *w, double *D)
{
  if (np < 2) return -1;
  const int N = np - 1;
  long double zl[64], pn[64];
  if (np > 64) return -1;
  zl[0] = -1.0L; zl[N] = 1.0L;
  for (int i = 1; i < N; i++) {
    /* Chebyshev-Gauss-Lobatto initial guess, then Newton on q(x) = P'_N(x). */
    long double x = -cosl(3.14159265358979323846264338327950288L * i / N);
    for (int it = 0; it < 100; it++) {
      long double p, dp;
      legendre_ld(N, x, &p, &dp);
      /* (1-x^2) P''_N = 2x P'_N - N(N+1) P_N */
      long double d2 = (2.0L * x * dp - N * (N + 1.0L) * p) / (1.0L - x * x);
      long double dx = dp / d2;
      x -= dx;
      if (fabsl(dx) < 1e-30L) break;
    }
    zl[i] = x;
  }
  /* symmetrise: z_i = -z_{N-i} exactly */
  for (int i = 0; i < np / 2; i++) {
    long double a = 0.5L * (zl[N - i] - zl[i]);
    zl[i] = -a; zl[N - i] = a;
  }
  if (np % 2) zl[N / 2] = 0.0L;
  for (int i = 0; i < np; i++) {
    long double dp;
    legendre_ld(N, zl[i], &pn[i], &dp);
    z[i] = (double)zl[i];
    w[i] = (double)(2.0L / (N * (N + 1.0L) * pn[i] * pn[i]));
  }
  for (int i = 0; i < np; i++)
    for (int j = 0; j < np; j++) {
      long double d;
      if (i != j) d = pn[i] / (pn[j] * (zl[i] - zl[j]));
      else if (i == 0) d = -N * (N + 1.0L) / 4.0L;
      else if (i == N) d = N * (N + 1.0L) / 4.0L;
      else d = 0.0L;
      D[i * np + j] = (double)d;
    }
  return 0;
}

/* Edge-major permutation: femlib/mapping.c:46-132 (dim == 2). */
void orc_edgemaps(int np, int *emap, int *pmap)
{
  int k = 0, n = 0;
  emap[0] = 0;
  for (int i = 1; i < np; i++) emap[++k] = n += 1;
  for (int i = 1; i < np; i++) emap[++k] = n += np;
  for (int i = 1; i < np; i++) emap[++k] = n -= 1;
  for (int i = 1; i < np; i++) emap[++k] = n -= np;
  for (int i = 1; i < np - 1; i++)
    for (int j = 1; j < np - 1; j++) emap[k++] = i * np + j;
  for (int i = 0; i < np * np; i++) pmap[emap[i]] = i;
}

/* Straight-sided element nodes: side points at GLL spacing, interior by the
 * Coons patch (src/mesh.cpp:772-886, straight sides of src/mesh.cpp:752-768).
 * vx/vy: the 4 vertices in CCW order. */
void orc_mesh_elmt(int np, const double *z, const double *vx, const double *vy,
                   double *x, double *y)
{
  const int nm = np - 1;
  double px[64], py[64], sp[64];
#define RMA(i, j) ((i) * np + (j))
  for (int s = 0; s < 4; s++) {
    const double x1 = vx[s], y1 = vy[s], x2 = vx[(s + 1) % 4], y2 = vy[(s + 1) % 4];
    const double dx = x2 - x1, dy = y2 - y1;
    for (int i = 0; i < np; i++) sp[i] = (s < 2) ? z[i] : -z[nm - i];
    for (int i = 0; i < np; i++) {
      px[i] = x1 + dx * 0.5 * (sp[i] + 1.0);
      py[i] = y1 + dy * 0.5 * (sp[i] + 1.0);
    }
    for (int i = 0; i < nm; i++) {
      int idx = (s == 0) ? RMA(0, i) : (s == 1) ? RMA(i, nm) : (s == 2) ? RMA(nm, nm - i) : RMA(nm - i, 0);
      x[idx] = px[i]; y[idx] = py[i];
    }
  }
  for (int i = 1; i < nm; i++)
    for (int j = 1; j < nm; j++) {
      const double *zr = z, *zs = z;
      x[RMA(i, j)] = 0.50 * ((1.0 - zr[j]) * x[RMA(i, 0)] + (1.0 + zr[j]) * x[RMA(i, nm)] +
                             (1.0 - zs[i]) * x[RMA(0, j)] + (1.0 + zs[i]) * x[RMA(nm, j)]) -
                     0.25 * ((1.0 - zr[j]) * (1.0 - zs[i]) * x[RMA(0, 0)] +
                             (1.0 - zr[j]) * (1.0 + zs[i]) * x[RMA(nm, 0)] +
                             (1.0 - zs[i]) * (1.0 + zr[j]) * x[RMA(0, nm)] +
                             (1.0 + zs[i]) * (1.0 + zr[j]) * x[RMA(nm, nm)]);
      y[RMA(i, j)] = 0.50 * ((1.0 - zr[j]) * y[RMA(i, 0)] + (1.0 + zr[j]) * y[RMA(i, nm)] +
                             (1.0 - zs[i]) * y[RMA(0, j)] + (1.0 + zs[i]) * y[RMA(nm, j)]) -
                     0.25 * ((1.0 - zr[j]) * (1.0 - zs[i]) * y[RMA(0, 0)] +
                             (1.0 - zr[j]) * (1.0 + zs[i]) * y[RMA(nm, 0)] +
                             (1.0 - zs[i]) * (1.0 + zr[j]) * y[RMA(0, nm)] +
                             (1.0 + zs[i]) * (1.0 + zr[j]) * y[RMA(nm, nm)]);
    }
#undef RMA
}

/* ------------------------------------------------------------------------ */
/* Mesh (Elements + NumberSys + boundary list)                               */
/* ------------------------------------------------------------------------ */

typedef struct {
  int np, npnp, next, nint, nel;
  int nglobal, nsolve_ns, nband;
  double *z, *w, *D, *DT;
  int *emap, *pmap;
  double *x, *y;                         /* nel*npnp */
  double *Q1, *Q2, *Q3, *Q4, *Q8;        /* nel*npnp */
  double *drdx, *drdy, *dsdx, *dsdy;     /* nel*npnp */
  int *hasQ3, *hasdrdx, *hasdrdy, *hasdsdx, *hasdsdy;
  int *btog, *bmask, *emask;             /* nel*next, nel */
  int nbound;
  int *b_elmt, *b_side, *b_kind;         /* kind: 0 essential, 1 natural, 2 mixed */
  double *b_K, *b_C;
  double *b_area;                        /* nbound*np */
  int mixed;
} orc_mesh;

static double dot_n(int n, const double *a, int ia, const double *b, int ib)
{
  double s = 0.0;
  for (int k = 0; k < n; k++) s += a[k * ia] * b[k * ib];
  return s;
}

/* C = A (m x k) * B (k x n), all row-major (veclib/blas.h:345-363 mxm). */
static void mxm(const double *A, int m, const double *B, int k, double *C, int n)
{
  for (int i = 0; i < m; i++)
    for (int j = 0; j < n; j++) {
      double s = 0.0;
      for (int p = 0; p < k; p++) s += A[i * k + p] * B[p * n + j];
      C[i * n + j] = s;
    }
}

/* C += A * B (veclib/blas.h mxma). */
static void mxma(const double *A, int m, const double *B, int k, double *C, int n)
{
  for (int i = 0; i < m; i++)
    for (int j = 0; j < n; j++) {
      double s = 0.0;
      for (int p = 0; p < k; p++) s += A[i * k + p] * B[p * n + j];
      C[i * n + j] += s;
    }
}

static double nrm2(int n, const double *a)
{
  double s = 0.0;
  for (int i = 0; i < n; i++) s += a[i] * a[i];
  return sqrt(s);
}

/* Element::mapping, src/element.cpp:1281-1436 (Cartesian, GLL). */
static int element_mapping(orc_mesh *M, int e)
{
  const int np = M->np, nn = M->npnp;
  const double *x = M->x + (size_t)e * nn, *y = M->y + (size_t)e * nn;
  double dxdr[256], dxds[256], dydr[256], dyds[256], jac[256], WW[256];
  double *Q1 = M->Q1 + (size_t)e * nn, *Q2 = M->Q2 + (size_t)e * nn, *Q3 = M->Q3 + (size_t)e * nn;
  double *Q4 = M->Q4 + (size_t)e * nn, *Q8 = M->Q8 + (size_t)e * nn;
  double *rx = M->drdx + (size_t)e * nn, *ry = M->drdy + (size_t)e * nn;
  double *sx = M->dsdx + (size_t)e * nn, *sy = M->dsdy + (size_t)e * nn;
  const double EPS = 4 * EPSDP;
  if (nn > 256) return -1;
  mxm(x, np, M->DT, np, dxdr, np);
  mxm(M->D, np, x, np, dxds, np);
  mxm(y, np, M->DT, np, dydr, np);
  mxm(M->D, np, y, np, dyds, np);
  double jmin = 1e300;
  for (int k = 0; k < nn; k++) {
    jac[k] = dxdr[k] * dyds[k] - dxds[k] * dydr[k];
    if (jac[k] < jmin) jmin = jac[k];
  }
  if (jmin < EPS) return -2; /* "Jacobian of element nonpositive" */
  for (int i = 0; i < np; i++)
    for (int j = 0; j < np; j++) WW[i * np + j] = M->w[i] * M->w[j];
  for (int k = 0; k < nn; k++) {
    Q1[k] = (dxds[k] * dxds[k] + dyds[k] * dyds[k]) / jac[k] * WW[k];
    Q2[k] = (dxdr[k] * dxdr[k] + dydr[k] * dydr[k]) / jac[k] * WW[k];
    Q3[k] = (-(dydr[k] * dyds[k]) - dxdr[k] * dxds[k]) / jac[k] * WW[k];
    Q4[k] = jac[k] * WW[k];
    Q8[k] = Q4[k];
    rx[k] = dyds[k] / jac[k];
    ry[k] = -dxds[k] / jac[k];
    sx[k] = -dydr[k] / jac[k];
    sy[k] = dxdr[k] / jac[k];
  }
  M->hasdrdx[e] = nrm2(nn, rx) >= EPS;
  M->hasdrdy[e] = nrm2(nn, ry) >= EPS;
  M->hasdsdx[e] = nrm2(nn, sx) >= EPS;
  M->hasdsdy[e] = nrm2(nn, sy) >= EPS;
  M->hasQ3[e] = nrm2(nn, Q3) >= EPS;
  if (!M->hasQ3[e]) memset(Q3, 0, sizeof(double) * nn);
  return 0;
}

/* Element::sideGeom, src/element.cpp:1653-1780: edge quadrature "area"
 * factor |dx/dr| w along the side, in CCW edge order. */
static void side_area(const orc_mesh *M, int e, int side, double *area)
{
  const int np = M->np, nn = M->npnp;
  const double *x = M->x + (size_t)e * nn, *y = M->y + (size_t)e * nn;
  int low, skip;
  switch (side) {
  case 0: low = 0; skip = 1; break;
  case 1: low = np - 1; skip = np; break;
  case 2: low = np * (np - 1); skip = 1; break;  /* derivative along r on row nm */
  default: low = 0; skip = np; break;            /* derivative along s on column 0 */
  }
  double xr[64], yr[64];
  for (int i = 0; i < np; i++) {
    xr[i] = dot_n(np, M->D + i * np, 1, x + low, skip);
    yr[i] = dot_n(np, M->D + i * np, 1, y + low, skip);
  }
  for (int i = 0; i < np; i++) {
    double a = sqrt(xr[i] * xr[i] + yr[i] * yr[i]) * M->w[i];
    area[i] = a;
  }
  /* Sides 2 and 3 are traversed with negative skip by the reference
   * (Veclib::copy with skip -1 / -np reverses the order of x,y but the area
   * is computed from the forward gemv and NOT reversed); GLL weights and
   * straight-side Jacobians are symmetric, so this is exact for the meshes
   * handled here.  Keep the reference's (unreversed) order.             */
}

orc_mesh *orc_mesh_create(int np, int nel, const double *x, const double *y,
                          const int *btog, const int *bmask, int nglobal, int nsolve, int nband,
                          int nbound, const int *b_elmt, const int *b_side, const int *b_kind,
                          const double *b_K, const double *b_C, int *info)
{
  orc_mesh *M = (orc_mesh *)calloc(1, sizeof(orc_mesh));
  const int nn = np * np, next = 4 * (np - 1);
  M->np = np; M->npnp = nn; M->next = next; M->nint = nn - next; M->nel = nel;
  M->nglobal = nglobal; M->nsolve_ns = nsolve; M->nband = nband;
  M->z = malloc(sizeof(double) * np); M->w = malloc(sizeof(double) * np);
  M->D = malloc(sizeof(double) * nn); M->DT = malloc(sizeof(double) * nn);
  M->emap = malloc(sizeof(int) * nn); M->pmap = malloc(sizeof(int) * nn);
  orc_gll(np, M->z, M->w, M->D);
  for (int i = 0; i < np; i++)
    for (int j = 0; j < np; j++) M->DT[j * np + i] = M->D[i * np + j];
  orc_edgemaps(np, M->emap, M->pmap);
  size_t tot = (size_t)nel * nn;
  M->x = malloc(sizeof(double) * tot); M->y = malloc(sizeof(double) * tot);
  memcpy(M->x, x, sizeof(double) * tot); memcpy(M->y, y, sizeof(double) * tot);
  double **arr[] = {&M->Q1, &M->Q2, &M->Q3, &M->Q4, &M->Q8, &M->drdx, &M->drdy, &M->dsdx, &M->dsdy};
  for (int k = 0; k < 9; k++) *arr[k] = calloc(tot, sizeof(double));
  int **iarr[] = {&M->hasQ3, &M->hasdrdx, &M->hasdrdy, &M->hasdsdx, &M->hasdsdy, &M->emask};
  for (int k = 0; k < 6; k++) *iarr[k] = calloc(nel, sizeof(int));
  M->btog = malloc(sizeof(int) * (size_t)nel * next);
  M->bmask = malloc(sizeof(int) * (size_t)nel * next);
  memcpy(M->btog, btog, sizeof(int) * (size_t)nel * next);
  memcpy(M->bmask, bmask, sizeof(int) * (size_t)nel * next);
  *info = 0;
  for (int e = 0; e < nel; e++) {
    int r = element_mapping(M, e);
    if (r) { *info = r; }
    int any = 0;
    for (int i = 0; i < next; i++) any |= bmask[e * next + i] != 0;
    M->emask[e] = any; /* src/bcmgr.cpp:799-803 */
  }
  M->nbound = nbound;
  M->b_elmt = malloc(sizeof(int) * (nbound + 1)); M->b_side = malloc(sizeof(int) * (nbound + 1));
  M->b_kind = malloc(sizeof(int) * (nbound + 1));
  M->b_K = malloc(sizeof(double) * (nbound + 1)); M->b_C = malloc(sizeof(double) * (nbound + 1));
  M->b_area = malloc(sizeof(double) * (size_t)(nbound + 1) * np);
  M->mixed = 0;
  for (int b = 0; b < nbound; b++) {
    M->b_elmt[b] = b_elmt[b]; M->b_side[b] = b_side[b]; M->b_kind[b] = b_kind[b];
    M->b_K[b] = b_K ? b_K[b] : 0.0; M->b_C[b] = b_C ? b_C[b] : 0.0;
    side_area(M, b_elmt[b], b_side[b], M->b_area + (size_t)b * np);
    if (b_kind[b] == 2) M->mixed = 1;
  }
  return M;
}

void orc_mesh_destroy(orc_mesh *M)
{
  if (!M) return;
  void *p[] = {M->z, M->w, M->D, M->DT, M->emap, M->pmap, M->x, M->y, M->Q1, M->Q2, M->Q3, M->Q4,
               M->Q8, M->drdx, M->drdy, M->dsdx, M->dsdy, M->hasQ3, M->hasdrdx, M->hasdrdy,
               M->hasdsdx, M->hasdsdy, M->btog, M->bmask, M->emask, M->b_elmt, M->b_side,
               M->b_kind, M->b_K, M->b_C, M->b_area};
  for (size_t k = 0; k < sizeof(p) / sizeof(p[0]); k++) free(p[k]);
  free(M);
}

/* Export geometry of element e (for product-vs-oracle checks). */
int orc_mesh_geom(const orc_mesh *M, int e, double *Q1, double *Q2, double *Q3, double *Q4, double *Q8)
{
  const size_t o = (size_t)e * M->npnp, n = M->npnp;
  memcpy(Q1, M->Q1 + o, n * 8); memcpy(Q2, M->Q2 + o, n * 8); memcpy(Q3, M->Q3 + o, n * 8);
  memcpy(Q4, M->Q4 + o, n * 8); memcpy(Q8, M->Q8 + o, n * 8);
  return M->hasQ3[e];
}

void orc_boundary_area(const orc_mesh *M, double *area) { memcpy(area, M->b_area, sizeof(double) * M->nbound * M->np); }

/* ------------------------------------------------------------------------ */
/* Element Helmholtz operators                                               */
/* ------------------------------------------------------------------------ */

/* Element::HelmholtzRow, src/element.cpp:1439-1509 (Cartesian; SVV off so
 * the SVV derivative matrices equal DV, src/svv.cpp:126-185).  Row (i,j) of
 * the elemental matrix into hij (np x np, row-major over (m,n)). */
static void helmholtz_row(const orc_mesh *M, int e, double hCon, int i, int j, double *hij)
{
  const int np = M->np, nn = M->npnp;
  const double *Q1 = M->Q1 + (size_t)e * nn, *Q2 = M->Q2 + (size_t)e * nn;
  const double *Q3 = M->Q3 + (size_t)e * nn, *Q4 = M->Q4 + (size_t)e * nn;
  const double *dt = M->DT, *dv = M->D;
  double work[64];
  memset(hij, 0, sizeof(double) * nn);
  for (int n = 0; n < np; n++) {
    for (int q = 0; q < np; q++) work[q] = dt[j * np + q] * dt[n * np + q];
    hij[i * np + n] = dot_n(np, Q1 + i * np, 1, work, 1);
  }
  for (int m = 0; m < np; m++) {
    for (int q = 0; q < np; q++) work[q] = dt[i * np + q] * dt[m * np + q];
    hij[m * np + j] += dot_n(np, Q2 + j, np, work, 1);
  }
  if (M->hasQ3[e])
    for (int m = 0; m < np; m++)
      for (int n = 0; n < np; n++) {
        hij[m * np + n] += Q3[i * np + n] * dv[n * np + j] * dv[i * np + m];
        hij[m * np + n] += Q3[m * np + j] * dv[j * np + n] * dv[m * np + i];
      }
  hij[i * np + j] += Q4[i * np + j] * hCon;
}

/* Full elemental matrix h (npnp x npnp, row-major, natural node order). */
void orc_element_matrix(const orc_mesh *M, int e, double hCon, double *h)
{
  const int np = M->np, nn = M->npnp;
  for (int i = 0; i < np; i++)
    for (int j = 0; j < np; j++) helmholtz_row(M, e, hCon, i, j, h + (size_t)(i * np + j) * nn);
}

/* Element::HelmholtzOp + HelmholtzKern, src/element.cpp:1564-1650 (Cartesian). */
static void helmholtz_op(const orc_mesh *M, int e, double hCon, const double *src, double *tgt)
{
  const int np = M->np, nn = M->npnp;
  const double *g1 = M->Q1 + (size_t)e * nn, *g2 = M->Q2 + (size_t)e * nn;
  const double *g3 = M->Q3 + (size_t)e * nn, *g4 = M->Q4 + (size_t)e * nn;
  double R[256], S[256], T[256];
  mxm(src, np, M->DT, np, R, np);
  mxm(M->D, np, src, np, S, np);
  if (M->hasQ3[e]) {
    for (int k = 0; k < nn; k++) {
      double tmp = R[k];
      R[k] = g1[k] * R[k] + g3[k] * S[k];
      S[k] = g2[k] * S[k] + g3[k] * tmp;
      T[k] = g4[k] * src[k] * hCon;
    }
  } else {
    for (int k = 0; k < nn; k++) {
      R[k] *= g1[k];
      S[k] *= g2[k];
      T[k] = g4[k] * src[k] * hCon;
    }
  }
  mxma(M->DT, np, S, np, T, np);
  mxma(R, np, M->D, np, T, np);
  memcpy(tgt, T, sizeof(double) * nn);
}

void orc_helmholtz_op(const orc_mesh *M, int e, double lambda2, double betak2, const double *src, double *tgt)
{
  helmholtz_op(M, e, betak2 + lambda2, src, tgt);
}

/* Element::HelmholtzDiag, src/element.cpp:1512-1561 (Cartesian), emap order. */
static void helmholtz_diag(const orc_mesh *M, int e, double hCon, double *diag)
{
  const int np = M->np, nn = M->npnp;
  const double *Q1 = M->Q1 + (size_t)e * nn, *Q2 = M->Q2 + (size_t)e * nn;
  const double *Q3 = M->Q3 + (size_t)e * nn, *Q4 = M->Q4 + (size_t)e * nn;
  const double *dt = M->DT, *dv = M->D;
  double dg[256], tmp[64];
  for (int i = 0, ij = 0; i < np; i++)
    for (int j = 0; j < np; j++, ij++) {
      for (int q = 0; q < np; q++) tmp[q] = dt[j * np + q] * dt[j * np + q];
      dg[ij] = dot_n(np, Q1 + i * np, 1, tmp, 1);
      for (int q = 0; q < np; q++) tmp[q] = dt[i * np + q] * dt[i * np + q];
      dg[ij] += dot_n(np, Q2 + j, np, tmp, 1);
      if (M->hasQ3[e]) dg[ij] += 2.0 * Q3[ij] * dv[j * np + j] * dv[i * np + i];
      dg[ij] += hCon * Q4[ij];
    }
  for (int k = 0; k < nn; k++) diag[k] = dg[M->emap[k]];
}

/* In-place inverse of a general n x n row-major matrix by LU with partial
 * pivoting (restates LAPACK dgetf2 + dgetri as used at
 * src/element.cpp:212-216).  Returns 0 or the 1-based singular pivot. */
static int lu_inverse(int n, double *A)
{
  int *piv = malloc(sizeof(int) * n);
  double *inv = calloc((size_t)n * n, sizeof(double));
  int info = 0;
  for (int k = 0; k < n; k++) {
    int p = k;
    double amax = fabs(A[k * n + k]);
    for (int i = k + 1; i < n; i++)
      if (fabs(A[i * n + k]) > amax) { amax = fabs(A[i * n + k]); p = i; }
    piv[k] = p;
    if (amax == 0.0) { info = k + 1; break; }
    if (p != k)
      for (int j = 0; j < n; j++) { double t = A[k * n + j]; A[k * n + j] = A[p * n + j]; A[p * n + j] = t; }
    for (int i = k + 1; i < n; i++) {
      double l = A[i * n + k] / A[k * n + k];
      A[i * n + k] = l;
      for (int j = k + 1; j < n; j++) A[i * n + j] -= l * A[k * n + j];
    }
  }
  if (!info) {
    /* Solve A X = P I column by column. */
    double *col = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    for (int c = 0; c < n; c++) {
      for (int i = 0; i < n; i++) col[i] = (i == c) ? 1.0 : 0.0;
      for (int k = 0; k < n; k++)
        if (piv[k] != k) { double t = col[k]; col[k] = col[piv[k]]; col[piv[k]] = t; }
      for (int i = 0; i < n; i++) {
        double s = col[i];
        for (int j = 0; j < i; j++) s -= A[i * n + j] * col[j];
        col[i] = s;
      }
      for (int i = n - 1; i >= 0; i--) {
        double s = col[i];
        for (int j = i + 1; j < n; j++) s -= A[i * n + j] * col[j];
        col[i] = s / A[i * n + i];
      }
      for (int i = 0; i < n; i++) inv[i * n + c] = col[i];
    }
    free(col);
    memcpy(A, inv, sizeof(double) * (size_t)n * n);
  }
  free(piv); free(inv);
  return info;
}

/* Element::HelmholtzSC, src/element.cpp:131-229.  Returns condensed hbb
 * (next x next), hbi <- hbi hii^-1 (next x nint), hii <- hii^-1. */
static int helmholtz_sc(const orc_mesh *M, int e, double hCon, double *hbb, double *hbi, double *hii)
{
  const int np = M->np, nn = M->npnp, next = M->next, nint = M->nint;
  double *rmat = malloc(sizeof(double) * nn), *rwrk = malloc(sizeof(double) * nn);
  for (int i = 0, ij = 0; i < np; i++)
    for (int j = 0; j < np; j++, ij++) {
      helmholtz_row(M, e, hCon, i, j, rmat);
      for (int k = 0; k < nn; k++) rwrk[k] = rmat[M->emap[k]];
      int eq = M->pmap[ij];
      if (eq < next) {
        memcpy(hbb + (size_t)eq * next, rwrk, sizeof(double) * next);
        memcpy(hbi + (size_t)eq * nint, rwrk + next, sizeof(double) * nint);
      } else
        memcpy(hii + (size_t)(eq - next) * nint, rwrk + next, sizeof(double) * nint);
    }
  free(rmat); free(rwrk);
  if (!nint) return 0;
  int info = lu_inverse(nint, hii);
  if (info) return info;
  double *t = malloc(sizeof(double) * (size_t)next * nint);
  mxm(hbi, next, hii, nint, t, nint);         /* Blas::mxm (hbi, hii) */
  /* Blas::mxmts: hbb -= t * hbi^T  (veclib/blas.h:375-378) */
  for (int i = 0; i < next; i++)
    for (int j = 0; j < next; j++) {
      double s = 0.0;
      for (int p = 0; p < nint; p++) s += t[i * nint + p] * hbi[j * nint + p];
      hbb[i * next + j] -= s;
    }
  memcpy(hbi, t, sizeof(double) * (size_t)next * nint);
  free(t);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* LAPACK band Cholesky (restated dpbtf2 "U") and band solve (dpbtrs "U").    */
/* Band storage: AB[j*ldab + kd + i - j] = A(i,j), max(0,j-kd) <= i <= j.     */
/* ------------------------------------------------------------------------ */

int orc_dpbtrf(int n, int kd, double *AB, int ldab)
{
  for (int j = 0; j < n; j++) {
    double *colj = AB + (size_t)j * ldab;
    double ajj = colj[kd];
    if (ajj <= 0.0) return j + 1;
    ajj = sqrt(ajj);
    colj[kd] = ajj;
    int kn = kd < n - j - 1 ? kd : n - j - 1;
    if (kn > 0) {
      /* row j, columns j+1..j+kn: A(j, j+c) at AB[(j+c)*ldab + kd - c] */
      for (int c = 1; c <= kn; c++) AB[(size_t)(j + c) * ldab + kd - c] /= ajj;
      /* trailing rank-1 update A(j+a, j+c) -= U(j,j+a) U(j,j+c), 1<=a<=c<=kn */
      for (int c = 1; c <= kn; c++) {
        const double ujc = AB[(size_t)(j + c) * ldab + kd - c];
        double *col = AB + (size_t)(j + c) * ldab;
        for (int a = 1; a <= c; a++) col[kd + a - c] -= AB[(size_t)(j + a) * ldab + kd - a] * ujc;
      }
    }
  }
  return 0;
}

void orc_dpbtrs(int n, int kd, const double *AB, int ldab, double *b)
{
  /* U^T y = b (forward), column-oriented dot products. */
  for (int j = 0; j < n; j++) {
    const double *colj = AB + (size_t)j * ldab;
    int i0 = j - kd > 0 ? j - kd : 0;
    double s = b[j];
    for (int i = i0; i < j; i++) s -= colj[kd + i - j] * b[i];
    b[j] = s / colj[kd];
  }
  /* U x = y (backward), column-oriented axpys. */
  for (int j = n - 1; j >= 0; j--) {
    const double *colj = AB + (size_t)j * ldab;
    b[j] /= colj[kd];
    const double xj = b[j];
    int i0 = j - kd > 0 ? j - kd : 0;
    for (int i = i0; i < j; i++) b[i] -= colj[kd + i - j] * xj;
  }
}

/* ------------------------------------------------------------------------ */
/* MatrixSys (src/matrix.cpp:139-317)                                         */
/* ------------------------------------------------------------------------ */

typedef struct {
  const orc_mesh *M;
  double lambda2, betak2;
  int method; /* 0 DIRECT, 1 JACPCG */
  int singular, nsolve, nglobal, nband, npts;
  double *H;          /* nsolve*nband */
  double *hbi, *hii;  /* nel*next*nint, nel*nint*nint */
  double *PC;         /* npts */
} orc_sys;

/* method: 0 DIRECT, 1 JACPCG, 2 DIRECT with the band assembled but not
 * factored (the caller factors it, e.g. with LAPACK dpbtrf as the reference
 * does at src/matrix.cpp:259, and hands it back with orc_sys_set_band). */
orc_sys *orc_sys_create(const orc_mesh *M, double lambda2, double betak2, int method, int *info)
{
  orc_sys *S = (orc_sys *)calloc(1, sizeof(orc_sys));
  const int next = M->next, nint = M->nint, nel = M->nel, np = M->np;
  const double hCon = betak2 + lambda2;
  const int factor = method == 0;
  if (method == 2) method = 0;
  S->M = M; S->lambda2 = lambda2; S->betak2 = betak2; S->method = method;
  S->nglobal = M->nglobal; S->nband = M->nband;
  /* src/matrix.cpp:166-169 */
  S->singular = (lambda2 + betak2) < EPSSP && (M->nglobal - M->nsolve_ns) == 0 && !M->mixed;
  S->nsolve = S->singular ? M->nsolve_ns - 1 : M->nsolve_ns;
  S->npts = M->nglobal + nel * nint;
  *info = 0;
  if (method == 0) {
    const int nsolve = S->nsolve, nband = S->nband;
    S->H = calloc((size_t)nsolve * nband + 1, sizeof(double));
    S->hbi = calloc((size_t)nel * next * nint + 1, sizeof(double));
    S->hii = calloc((size_t)nel * nint * nint + 1, sizeof(double));
    double *hbb = malloc(sizeof(double) * next * next);
    for (int e = 0; e < nel; e++) {
      int r = helmholtz_sc(M, e, hCon, hbb, S->hbi + (size_t)e * next * nint, S->hii + (size_t)e * nint * nint);
      if (r) { *info = -1000 - e; free(hbb); return S; }
      const int *bmap = M->btog + (size_t)e * next;
      for (int i = 0; i < next; i++) {
        int m = bmap[i];
        if (m >= nsolve) continue;
        for (int k = 0; k < next; k++) {
          int n = bmap[k];
          if (n < nsolve && n >= m) {
            if (n - m >= nband) { *info = -2; free(hbb); return S; }
            S->H[(size_t)n * nband + (nband - 1) + m - n] += hbb[i * next + k];
          }
        }
      }
    }
    free(hbb);
    /* Mixed BC diagonal terms: Mixed::augmentSC, src/condition.cpp:347-381 */
    for (int b = 0; b < M->nbound; b++) {
      if (M->b_kind[b] != 2) continue;
      const int nm = np - 1, side = M->b_side[b];
      const int *bmap = M->btog + (size_t)M->b_elmt[b] * next;
      const int *start = bmap + side * nm;
      const double *area = M->b_area + (size_t)b * np;
      for (int i = 0; i < nm; i++) {
        int k = start[i];
        if (k < nsolve) S->H[(size_t)k * nband + nband - 1] += M->b_K[b] * area[i];
      }
      int i = (side == 3) ? bmap[0] : start[nm];
      if (i < nsolve) S->H[(size_t)i * nband + nband - 1] += M->b_K[b] * area[nm];
    }
    if (nsolve && factor) {
      int r = orc_dpbtrf(nsolve, nband - 1, S->H, nband);
      if (r) *info = r;
    }
  } else {
    /* JACPCG diagonal, src/matrix.cpp:276-317 */
    S->PC = calloc(S->npts, sizeof(double));
    for (int b = 0; b < M->nbound; b++) {
      if (M->b_kind[b] != 2) continue;
      const int nm = np - 1, side = M->b_side[b];
      const int *bmap = M->btog + (size_t)M->b_elmt[b] * next;
      const int *start = bmap + side * nm;
      const double *area = M->b_area + (size_t)b * np;
      for (int i = 0; i < nm; i++) S->PC[start[i]] += M->b_K[b] * area[i];
      int i = (side == 3) ? bmap[0] : start[nm];
      S->PC[i] += M->b_K[b] * area[nm];
    }
    double ed[256];
    double *PCi = S->PC + M->nglobal;
    for (int e = 0; e < nel; e++, PCi += nint) {
      helmholtz_diag(M, e, hCon, ed);
      const int *bmap = M->btog + (size_t)e * next;
      for (int i = 0; i < next; i++) S->PC[bmap[i]] += ed[i];
      memcpy(PCi, ed + next, sizeof(double) * nint);
    }
    for (int i = 0; i < S->npts; i++) S->PC[i] = 1.0 / S->PC[i];
  }
  return S;
}

void orc_sys_destroy(orc_sys *S)
{
  if (!S) return;
  free(S->H); free(S->hbi); free(S->hii); free(S->PC);
  free(S);
}

int orc_sys_nsolve(const orc_sys *S) { return S->nsolve; }
int orc_sys_singular(const orc_sys *S) { return S->singular; }
void orc_sys_band(const orc_sys *S, double *H) { memcpy(H, S->H, sizeof(double) * (size_t)S->nsolve * S->nband); }
void orc_sys_set_band(orc_sys *S, const double *H) { memcpy(S->H, H, sizeof(double) * (size_t)S->nsolve * S->nband); }
void orc_sys_hbi(const orc_sys *S, double *hbi)
{
  memcpy(hbi, S->hbi, sizeof(double) * (size_t)S->M->nel * S->M->next * S->M->nint);
}
void orc_sys_hii(const orc_sys *S, double *hii)
{
  memcpy(hii, S->hii, sizeof(double) * (size_t)S->M->nel * S->M->nint * S->M->nint);
}
void orc_sys_pc(const orc_sys *S, double *pc) { memcpy(pc, S->PC, sizeof(double) * S->npts); }

/* ------------------------------------------------------------------------ */
/* Field::solve helpers, src/field.cpp:728-1040                               */
/* ------------------------------------------------------------------------ */

/* Essential::set (src/condition.cpp:80-101) for every essential boundary:
 * Field::getEssential, src/field.cpp:994-1019. */
static void get_essential(const orc_mesh *M, const double *bc, double *tgt)
{
  const int np = M->np, nm = np - 1, next = M->next;
  for (int b = 0; b < M->nbound; b++) {
    if (M->b_kind[b] != 0) continue;
    const double *src = bc + (size_t)b * np;
    const int *bmap = M->btog + (size_t)M->b_elmt[b] * next;
    const int side = M->b_side[b];
    const int *start = bmap + side * nm;
    for (int i = 0; i < nm; i++) tgt[start[i]] = src[i];
    if (side == 3) tgt[bmap[0]] = src[nm];
    else tgt[start[nm]] = src[nm];
  }
}

/* Natural::sum / Mixed::sum (src/condition.cpp:192-219, 297-323). */
static void sum_natural(const orc_mesh *M, const double *bc, double *tgt)
{
  const int np = M->np, nm = np - 1, next = M->next;
  double work[64];
  for (int b = 0; b < M->nbound; b++) {
    const int kind = M->b_kind[b];
    if (kind == 0) continue;
    const double *src = bc + (size_t)b * np;
    const double *area = M->b_area + (size_t)b * np;
    const int *bmap = M->btog + (size_t)M->b_elmt[b] * next;
    const int side = M->b_side[b];
    const int *start = bmap + side * nm;
    if (kind == 1) for (int i = 0; i < np; i++) work[i] = src[i] * area[i];
    else for (int i = 0; i < np; i++) work[i] = (M->b_K[b] * M->b_C[b]) * area[i];
    for (int i = 0; i < nm; i++) tgt[start[i]] += work[i];
    if (side == 3) tgt[bmap[0]] += work[nm];
    else tgt[start[nm]] += work[nm];
  }
}

/* Mixed::augmentOp (src/condition.cpp:384-410). */
static void augment_op(const orc_mesh *M, const double *x, double *y)
{
  const int np = M->np, nm = np - 1, next = M->next;
  for (int b = 0; b < M->nbound; b++) {
    if (M->b_kind[b] != 2) continue;
    const double *area = M->b_area + (size_t)b * np;
    const int *bmap = M->btog + (size_t)M->b_elmt[b] * next;
    const int side = M->b_side[b];
    const int *start = bmap + side * nm;
    for (int i = 0; i < nm; i++) y[start[i]] += M->b_K[b] * area[i] * x[start[i]];
    int i = (side == 3) ? bmap[0] : start[nm];
    y[i] += M->b_K[b] * area[nm] * x[i];
  }
}

/* Field::constrain, src/field.cpp:728-768: force <- -(M f + H g). */
static void constrain(const orc_mesh *M, double hCon, double *force, const double *esstlbc)
{
  const int nn = M->npnp, next = M->next, nel = M->nel;
  double u[256];
  for (int e = 0; e < nel; e++) {
    double *f = force + (size_t)e * nn;
    const double *Q8 = M->Q8 + (size_t)e * nn;
    for (int k = 0; k < nn; k++) f[k] *= Q8[k];
    if (M->emask[e]) {
      memset(u, 0, sizeof(double) * nn);
      const int *btog = M->btog + (size_t)e * next;
      for (int i = 0; i < next; i++) u[M->emap[i]] = esstlbc[btog[i]];
      helmholtz_op(M, e, hCon, u, u);
      for (int k = 0; k < nn; k++) f[k] += u[k];
    }
  }
  for (size_t k = 0; k < (size_t)nel * nn; k++) force[k] = -force[k];
}

/* Field::HelmholtzOperator, src/field.cpp:771-856 (non-vector branch). */
static void global_op(const orc_sys *S, const double *x, double *y)
{
  const orc_mesh *M = S->M;
  const int nn = M->npnp, next = M->next, nint = M->nint;
  const double hCon = S->betak2 + S->lambda2;
  double P[256];
  memset(y, 0, sizeof(double) * S->npts);
  if (M->mixed) augment_op(M, x, y);
  for (int e = 0; e < M->nel; e++) {
    const int *gid = M->btog + (size_t)e * next;
    const double *xint = x + M->nglobal + (size_t)e * nint;
    double *yint = y + M->nglobal + (size_t)e * nint;
    for (int i = 0; i < next; i++) P[M->emap[i]] = x[gid[i]];
    for (int i = 0; i < nint; i++) P[M->emap[next + i]] = xint[i];
    helmholtz_op(M, e, hCon, P, P);
    for (int i = 0; i < next; i++) y[gid[i]] += P[M->emap[i]];
    for (int i = 0; i < nint; i++) yint[i] += P[M->emap[next + i]];
  }
}

void orc_global_op(const orc_sys *S, const double *x, double *y) { global_op(S, x, y); }

/* Field::setEssential + Element::bndryMask (src/field.cpp:1022-1040,
 * src/element.cpp:501-537). */
static void set_essential(const orc_mesh *M, const double *src, double *tgt)
{
  const int nn = M->npnp, next = M->next;
  for (int e = 0; e < M->nel; e++) {
    if (!M->emask[e]) continue;
    const int *bmsk = M->bmask + (size_t)e * next, *btog = M->btog + (size_t)e * next;
    double *t = tgt + (size_t)e * nn;
    for (int i = 0; i < next; i++)
      if (bmsk[i]) t[M->emap[i]] = src[btog[i]];
  }
}

/* Field::solve for ONE data plane, src/field.cpp:509-725.
 *   unknown : plane of element data (in: initial guess, out: solution)
 *   forcing : plane of element data, overwritten (as in the reference)
 *   bc      : nbound*np boundary-line values for this plane
 * Returns PCG iteration count (JACPCG) or 0 (DIRECT); <0 on error. */
int orc_solve_plane(const orc_sys *S, double *unknown, double *forcing, const double *bc,
                    double tol_rel, int step_max)
{
  const orc_mesh *M = S->M;
  const int nn = M->npnp, next = M->next, nint = M->nint, nel = M->nel;
  const int nglobal = S->nglobal, nsolve = S->nsolve, nzero = nglobal - nsolve;
  const double hCon = S->betak2 + S->lambda2;
  if (S->method == 0) {
    double *RHS = calloc(nglobal + 1, sizeof(double));
    double work[256];
    get_essential(M, bc, RHS);
    constrain(M, hCon, forcing, RHS);
    /* Field::buildRHS (direct branch), src/field.cpp:859-925 */
    memset(RHS, 0, sizeof(double) * nglobal);
    for (int e = 0; e < nel; e++) {
      double *F = forcing + (size_t)e * nn;
      const int *btog = M->btog + (size_t)e * next;
      const double *hbi = S->hbi + (size_t)e * next * nint;
      /* Element::local2globalSumSC, src/element.cpp:356-395 */
      for (int k = 0; k < nn; k++) work[k] = F[M->emap[k]];
      memcpy(F, work, sizeof(double) * nn);
      for (int b = 0; b < next; b++) F[b] -= dot_n(nint, hbi + (size_t)b * nint, 1, F + next, 1);
      for (int b = 0; b < next; b++) RHS[btog[b]] += F[b];
    }
    sum_natural(M, bc, RHS);
    memset(RHS + nsolve, 0, sizeof(double) * nzero);
    if (nsolve) orc_dpbtrs(nsolve, S->nband - 1, S->H, S->nband, RHS);
    /* Element::global2localSC, src/element.cpp:398-438 */
    for (int e = 0; e < nel; e++) {
      double *F = forcing + (size_t)e * nn, *tgt = unknown + (size_t)e * nn;
      const int *btog = M->btog + (size_t)e * next;
      const double *hbi = S->hbi + (size_t)e * next * nint;
      const double *hii = S->hii + (size_t)e * nint * nint;
      for (int b = 0; b < next; b++) work[b] = RHS[btog[b]];
      for (int b = 0; b < next; b++) tgt[M->emap[b]] = work[b];
      if (nint) {
        double *Fi = F + next, wint[256];
        memcpy(wint, Fi, sizeof(double) * nint);
        for (int r = 0; r < nint; r++) Fi[r] = dot_n(nint, hii + (size_t)r * nint, 1, wint, 1);
        for (int r = 0; r < nint; r++) Fi[r] -= dot_n(next, hbi + r, nint, work, 1);
        for (int r = 0; r < nint; r++) tgt[M->emap[next + r]] = Fi[r];
      }
    }
    memset(RHS, 0, sizeof(double) * nglobal);
    get_essential(M, bc, RHS);
    set_essential(M, RHS, unknown);
    free(RHS);
    return 0;
  }
  /* JACPCG, src/field.cpp:627-720 */
  const int npts = S->npts;
  double *r = calloc(npts, sizeof(double)), *p = calloc(npts, sizeof(double));
  double *q = calloc(npts, sizeof(double)), *x = calloc(npts, sizeof(double));
  double *z = calloc(npts, sizeof(double));
  get_essential(M, bc, x);
  constrain(M, hCon, forcing, x);
  /* buildRHS, iterative branch */
  memset(r, 0, sizeof(double) * npts);
  for (int e = 0; e < nel; e++) {
    const double *F = forcing + (size_t)e * nn;
    const int *gid = M->btog + (size_t)e * next;
    double *rint = r + nglobal + (size_t)e * nint;
    for (int i = 0; i < next; i++) r[gid[i]] += F[M->emap[i]];
    for (int i = 0; i < nint; i++) rint[i] += F[M->emap[next + i]];
  }
  sum_natural(M, bc, r);
  memset(r + nsolve, 0, sizeof(double) * nzero);
  double epsb2 = tol_rel * sqrt(dot_n(npts, r, 1, r, 1));
  epsb2 *= epsb2;
  /* Field::local2global of the initial guess */
  for (int e = 0; e < nel; e++) {
    const double *src = unknown + (size_t)e * nn;
    const int *gid = M->btog + (size_t)e * next;
    double *xint = x + nglobal + (size_t)e * nint;
    for (int i = 0; i < next; i++) x[gid[i]] = src[M->emap[i]];
    for (int i = 0; i < nint; i++) xint[i] = src[M->emap[next + i]];
  }
  memset(x + nsolve, 0, sizeof(double) * nzero);
  memcpy(q, x, sizeof(double) * npts);
  global_op(S, q, p);
  memset(p + nsolve, 0, sizeof(double) * nzero);
  memset(r + nsolve, 0, sizeof(double) * nzero);
  for (int i = 0; i < npts; i++) r[i] -= p[i];
  double r2 = dot_n(npts, r, 1, r, 1), rho1 = 0.0, rho2 = 1.0;
  int it = 0;
  while (r2 > epsb2 && ++it < step_max) {
    for (int i = 0; i < npts; i++) z[i] = S->PC[i] * r[i];
    rho1 = dot_n(npts, r, 1, z, 1);
    if (it == 1) memcpy(p, z, sizeof(double) * npts);
    else {
      double beta = rho1 / rho2;
      for (int i = 0; i < npts; i++) p[i] = beta * p[i] + z[i];
    }
    global_op(S, p, q);
    memset(q + nsolve, 0, sizeof(double) * nzero);
    double dotp = dot_n(npts, p, 1, q, 1);
    double alpha = rho1 / dotp;
    for (int i = 0; i < npts; i++) x[i] += alpha * p[i];
    for (int i = 0; i < npts; i++) r[i] -= alpha * q[i];
    rho2 = rho1;
    r2 = dot_n(npts, r, 1, r, 1);
  }
  /* Field::global2local, then essential BCs */
  for (int e = 0; e < nel; e++) {
    double *tgt = unknown + (size_t)e * nn;
    const int *gid = M->btog + (size_t)e * next;
    const double *xint = x + nglobal + (size_t)e * nint;
    for (int i = 0; i < next; i++) tgt[M->emap[i]] = x[gid[i]];
    for (int i = 0; i < nint; i++) tgt[M->emap[next + i]] = xint[i];
  }
  memset(x, 0, sizeof(double) * nglobal);
  get_essential(M, bc, x);
  set_essential(M, x, unknown);
  free(r); free(p); free(q); free(x); free(z);
  return it;
}
