// sx_factor.cu -- GPU set-up of a DIRECT or JACPCG system (MatrixSys).
//
// DIRECT (src/matrix.cpp:175-274):
//   1. k_elem_condense: one CTA per element builds the elemental Helmholtz
//      matrix in edge-major order (Element::HelmholtzRow,
//      src/element.cpp:1439-1509), inverts the interior block (the reference
//      uses getrf+getri, src/element.cpp:212-216; hii is SPD here so
//      Gauss-Jordan without pivoting is used) and condenses
//      hbb -= hbi hii^-1 hib, hbi <- hbi hii^-1 (src/element.cpp:218-220).
//   2. k_band_add: direct-stiffness assembly of hbb into the banded matrix,
//      one element colour per launch so no two CTAs touch the same entry
//      (deterministic; src/matrix.cpp:236-241).  Mixed-BC diagonal terms
//      follow in boundary order (Mixed::augmentSC, src/condition.cpp:347-381).
//   3. Tiled right-looking banded Cholesky, A = U^T U (LAPACK dpbtrf "U",
//      src/matrix.cpp:259): per block column k, k_potrf factors the diagonal
//      tile and forms its inverse, k_trsm forms the off-diagonal tiles of
//      block row k, k_update applies the trailing rank-nb update inside the
//      band.  All systems of a batch share each launch.
// JACPCG (src/matrix.cpp:276-317): k_elem_diag + k_diag_dss.
#include <cmath>
#include <cstring>
#include <mutex>

#include "sx_internal.h"
#include "sx_kernels.cuh"
#include "sx_ptx.cuh"

namespace sx {

// ---------------------------------------------------------------------------
// Element matrix + static condensation
// ---------------------------------------------------------------------------

// smem (doubles): D nn | Q1..Q4 4nn | hbb next^2 | hbi next*nint | hii nint^2 |
// t next*nint | colk nint ; ints: emap nn
static size_t condense_smem_np(int np) {
  const size_t nn = (size_t)np * np, ne = 4 * (size_t)(np - 1), ni = nn - ne;
  return sizeof(double) * (5 * nn + ne * ne + 2 * ne * ni + ni * ni + ni) + sizeof(int) * nn + 16;
}
static size_t condense_smem(const MeshView &M) { return condense_smem_np(M.np); }

__global__ void k_elem_condense(MeshView M, double hCon, double *__restrict__ hbi_out,
                                double *__restrict__ hii_out, double *__restrict__ hbb_out,
                                int *status) {
  extern __shared__ double sm[];
  const int np = M.np, nn = M.npnp, next = M.next, nint = M.nint;
  const int e = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  double *D = sm, *Q1 = D + nn, *Q2 = Q1 + nn, *Q3 = Q2 + nn, *Q4 = Q3 + nn;
  double *hbb = Q4 + nn, *hbi = hbb + next * next, *hii = hbi + next * nint;
  double *t = hii + nint * nint, *colk = t + next * nint;
  int *emap = (int *)(colk + nint);
  __shared__ int bad;
  if (tid == 0) bad = 0;
  const size_t eo = (size_t)e * nn;
  for (int i = tid; i < nn; i += nt) {
    D[i] = M.D[i];
    Q1[i] = M.Q1[eo + i];
    Q2[i] = M.Q2[eo + i];
    Q3[i] = M.Q3[eo + i];
    Q4[i] = M.Q4[eo + i];
    emap[i] = M.emap[i];
  }
  __syncthreads();
  const bool q3 = M.hasQ3[e];
  // Entry H[(i,j),(m,n)] of the elemental matrix, accumulated in the order
  // of HelmholtzRow: Q1 term, Q2 term, the two Q3 terms, then Q4*hCon.
  for (int idx = tid; idx < nn * nn; idx += nt) {
    const int a = idx / nn, b = idx - a * nn;
    if (a >= next && b < next) continue;
    const int r = emap[a], c = emap[b];
    const int i = r / np, j = r - i * np, m = c / np, n = c - m * np;
    double h = 0.0;
    if (m == i) {
      double s = 0.0;
      for (int q = 0; q < np; q++) s += Q1[i * np + q] * (D[q * np + j] * D[q * np + n]);
      h = s;
    }
    if (n == j) {
      double s = 0.0;
      for (int p = 0; p < np; p++) s += Q2[p * np + j] * (D[p * np + i] * D[p * np + m]);
      h += s;
    }
    if (q3) {
      h += Q3[i * np + n] * D[n * np + j] * D[i * np + m];
      h += Q3[m * np + j] * D[j * np + n] * D[m * np + i];
    }
    if (m == i && n == j) h += Q4[i * np + j] * hCon;
    if (a < next) {
      if (b < next)
        hbb[a * next + b] = h;
      else
        hbi[a * nint + (b - next)] = h;
    } else {
      hii[(a - next) * nint + (b - next)] = h;
    }
  }
  __syncthreads();
  // In-place Gauss-Jordan inverse of the SPD interior block.
  for (int k = 0; k < nint; k++) {
    const double p = hii[k * nint + k];
    for (int i = tid; i < nint; i += nt) colk[i] = hii[i * nint + k];
    // a zero (or NaN) pivot: hii is singular (src/element.cpp:212-216); a
    // negative one: hii, a principal block of H, is not positive definite,
    // so neither is H -- the reference's getrf/getri go on with an
    // indefinite hii and its dpbtrf then fails (src/matrix.cpp:259-261)
    if (tid == 0) bad |= (p < 0.0) ? 2 : (!(p > 0.0) ? 1 : 0);
    __syncthreads();
    const double rp = (p != 0.0 && p == p) ? 1.0 / p : 1.0;
    for (int j = tid; j < nint; j += nt) hii[k * nint + j] = ((j == k) ? 1.0 : hii[k * nint + j]) * rp;
    __syncthreads();
    for (int idx = tid; idx < nint * nint; idx += nt) {
      const int i = idx / nint, j = idx - i * nint;
      if (i == k) continue;
      const double v = (j == k) ? 0.0 : hii[idx];
      hii[idx] = v - colk[i] * hii[k * nint + j];
    }
    __syncthreads();
  }
  // t = hbi * hii^-1 ; hbb -= t * hbi^T
  for (int idx = tid; idx < next * nint; idx += nt) {
    const int b = idx / nint, c = idx - b * nint;
    double s = 0.0;
    for (int q = 0; q < nint; q++) s += hbi[b * nint + q] * hii[q * nint + c];
    t[idx] = s;
  }
  __syncthreads();
  for (int idx = tid; idx < next * next; idx += nt) {
    const int b = idx / next, b2 = idx - b * next;
    double s = 0.0;
    for (int q = 0; q < nint; q++) s += t[b * nint + q] * hbi[b2 * nint + q];
    hbb[idx] -= s;
  }
  __syncthreads();
  double *ob = hbi_out + (size_t)e * next * nint;
  for (int i = tid; i < next * nint; i += nt) ob[i] = t[i];
  double *oi = hii_out + (size_t)e * nint * nint;
  // column-major, (r, c) at c * nint + r: the back-substitution's threads
  // own rows and read a column per step
  for (int o = tid; o < nint * nint; o += nt) {
    const int c = o / nint, r = o - c * nint;
    oi[o] = hii[r * nint + c];
  }
  double *oh = hbb_out + (size_t)e * next * next;
  for (int i = tid; i < next * next; i += nt) oh[i] = hbb[i];
  if (tid == 0 && bad)
    atomicOr(status, ((bad & 1) ? 1 << SX_ERR_SINGULAR_HII : 0) | ((bad & 2) ? 1 << SX_ERR_NOT_SPD : 0));
}

// ---------------------------------------------------------------------------
// Band assembly into tiles
// ---------------------------------------------------------------------------

__global__ void k_band_identity_pad(double *tiles, int J, int nsolve, int nblk) {
  const int g = nsolve + blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nblk * NB) return;
  const int b = g / NB, r = g - b * NB;
  tiles[((size_t)b * (J + 1)) * TSZ + (size_t)r * LDT + r] = 1.0;
}

__global__ void k_band_add(MeshView M, const int *__restrict__ elems, const double *__restrict__ hbb,
                           double *tiles, int J, int nsolve, int *status) {
  const int e = elems[blockIdx.x];
  const int next = M.next, kd = M.nband - 1;
  const int *bt = M.btog + (size_t)e * next;
  const double *h = hbb + (size_t)e * next * next;
  for (int idx = threadIdx.x; idx < next * next; idx += blockDim.x) {
    const int i = idx / next, k = idx - i * next;
    const int m = bt[i], n = bt[k];
    if (m < nsolve && n < nsolve && n >= m) {
      if (n - m > kd) {
        atomicOr(status, 1 << SX_ERR_BAND);
        continue;
      }
      tiles[tile_addr(m, n, J)] += h[idx];
    }
  }
}

// Mixed::augmentSC in boundary order (one thread: tiny, order-preserving).
__global__ void k_band_mixed(MeshView M, double *tiles, int J, int nsolve) {
  if (threadIdx.x || blockIdx.x) return;
  const int np = M.np, nm = np - 1;
  for (int b = 0; b < M.nbound; b++) {
    if (M.b_kind[b] != SX_BC_MIXED) continue;
    const int *bmap = M.btog + (size_t)M.b_elmt[b] * M.next;
    const int side = M.b_side[b];
    const double K = M.b_K[b];
    const double *area = M.b_area + (size_t)b * np;
    for (int i = 0; i < nm; i++) {
      const int k = bmap[side * nm + i];
      if (k < nsolve) tiles[tile_addr(k, k, J)] += K * area[i];
    }
    const int i = (side == 3) ? bmap[0] : bmap[side * nm + nm];
    if (i < nsolve) tiles[tile_addr(i, i, J)] += K * area[nm];
  }
}

// ---------------------------------------------------------------------------
// Tiled banded Cholesky
// ---------------------------------------------------------------------------

__device__ __forceinline__ void tile_load(double *dst, const double *__restrict__ src) {
  const double2 *s = reinterpret_cast<const double2 *>(src);
  double2 *d = reinterpret_cast<double2 *>(dst);
  for (int i = threadIdx.x; i < TSZ / 2; i += blockDim.x) d[i] = s[i];
}

__device__ __forceinline__ void tile_store(double *dst, const double *src) {
  const double2 *s = reinterpret_cast<const double2 *>(src);
  double2 *d = reinterpret_cast<double2 *>(dst);
  for (int i = threadIdx.x; i < TSZ / 2; i += blockDim.x) d[i] = s[i];
}

// Factor the diagonal tile of block column k and store its inverse.
// Factor the diagonal tile of block column k, A = U^T U (upper), and form
// D_k = U^-1, one CTA of 256 threads per system.
//   Cholesky, right-looking: thread t owns column j = t % 64 at rows i = t /
//   64 (mod 4).  Step c takes d = sqrt(A[c][c]), r = 1/d (every thread, from
//   the same shared value) and updates A[i][j] -= (A[c][i] r)(A[c][j] r)
//   for c < i <= j; row c itself is scaled by its owners at step c + 1, when
//   no thread reads it any more.  One barrier per step.
//   Inverse, by rows from the bottom: X[i][i] = 1/U[i][i], X[i][j] =
//   -(sum_{l=i+1..j} U[i][l] X[l][j]) / U[i][i]; four consecutive lanes
//   split each sum and combine it with two shuffles.  One barrier per row.
__global__ void __launch_bounds__(256) k_potrf(const SysDesc *__restrict__ sys, int k) {
  const SysDesc S = sys[blockIdx.x];
  if (k >= S.nblk) return;
  extern __shared__ __align__(16) double smp[];
  double *A = smp, *X = smp + TSZ;
  __shared__ int bad;
  const int tid = threadIdx.x;
  double *T = S.tiles + ((size_t)k * (S.J + 1)) * TSZ;
  if (tid == 0) bad = 0;
  tile_load(A, T);
  for (int idx = tid; idx < TSZ; idx += 256) X[idx] = 0.0;
  __syncthreads();
  const int j = tid & (NB - 1), rg = tid >> 6;
  double d_prev = 1.0, r_prev = 1.0;
  for (int c = 0; c < NB; c++) {
    double a = A[c * LDT + c];
    if (!(a > 0.0)) {
      if (tid == 0) bad = 1;
      a = 1.0;
    }
    const double d = sqrt(a), r = 1.0 / d;
    // row c - 1 is final: its owners scale it (and set its diagonal)
    if (c > 0 && ((c - 1) & 3) == rg && j >= c - 1)
      A[(c - 1) * LDT + j] = j == c - 1 ? d_prev : A[(c - 1) * LDT + j] * r_prev;
    if (j > c) {
      const double ucj = A[c * LDT + j] * r;
      for (int i = c + 1 + ((rg - (c + 1)) & 3); i <= j; i += 4) A[i * LDT + j] -= (A[c * LDT + i] * r) * ucj;
    }
    d_prev = d;
    r_prev = r;
    __syncthreads();
  }
  if (rg == ((NB - 1) & 3) && j == NB - 1) A[(NB - 1) * LDT + NB - 1] = d_prev;
  __syncthreads();
  for (int idx = tid; idx < NB * NB; idx += 256) {
    const int ii = idx / NB, jj = idx % NB;
    if (jj < ii) A[ii * LDT + jj] = 0.0;
  }
  __syncthreads();
  tile_store(T, A);
  const int jc = tid >> 2, q = tid & 3;
  for (int i = NB - 1; i >= 0; i--) {
    double s = 0.0;
    if (jc > i)
      for (int l = i + 1 + q; l <= jc; l += 4) s += A[i * LDT + l] * X[l * LDT + jc];
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    if (q == 0 && jc >= i) X[i * LDT + jc] = jc == i ? 1.0 / A[i * LDT + i] : -s / A[i * LDT + i];
    __syncthreads();
  }
  tile_store(S.dinv + (size_t)k * TSZ, X);
  if (tid == 0 && bad) atomicOr(S.status, 1 << SX_ERR_NOT_SPD);
}

// Tile products on the FP64 tensor cores (mma.sync m8n8k4, f64).  The two
// factor tiles of a product are staged into shared memory with rows padded
// to LDM = 68 doubles (68 = 4 mod 16: the 4 x 8 slab a fragment reads, rows
// t = 0..3 and columns g = 0..7, falls on 16 distinct bank pairs in each
// half-warp).  Warp w owns rows 16 (w / 2) .. +16 and columns 32 (w % 2) ..
// +32 of the 64 x 64 result: 2 x 4 blocks of 8 x 8, two accumulators a
// thread each, held in registers from the first product to the store.
constexpr int LDM = NB + 4;

__device__ __forceinline__ void tile_stage_mma(double *dst, const double *__restrict__ src) {
  for (int idx = threadIdx.x; idx < NB * NB; idx += blockDim.x) {
    const int r = idx >> 6, c = idx & (NB - 1);
    cp_async8_ca(dst + r * LDM + c, src + r * LDT + c);
  }
}

struct MmaAcc {
  double v[2][4][2];
};

// This thread's result elements: (row r0 + 8m + g, column c0 + 8n + 2t + q).
__device__ __forceinline__ void mma_coords(int &r0, int &c0, int &g, int &t) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  g = lane >> 2;
  t = lane & 3;
  r0 = (w >> 1) * 16;
  c0 = (w & 1) * 32;
}

__device__ __forceinline__ void mma_f64(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// acc += (neg ? -1 : 1) * A^T B over the NB rows of the staged tiles:
// entry (r, c) gains sum_l A[l][r] B[l][c].
__device__ __forceinline__ void mma_tn(MmaAcc &acc, const double *As, const double *Bs, bool neg) {
  int r0, c0, g, t;
  mma_coords(r0, c0, g, t);
#pragma unroll 4
  for (int l0 = 0; l0 < NB; l0 += 4) {
    const double *Ar = As + (l0 + t) * LDM + r0 + g, *Br = Bs + (l0 + t) * LDM + c0 + g;
    double a[2], b[4];
#pragma unroll
    for (int m = 0; m < 2; m++) a[m] = neg ? -Ar[8 * m] : Ar[8 * m];
#pragma unroll
    for (int n = 0; n < 4; n++) b[n] = Br[8 * n];
#pragma unroll
    for (int m = 0; m < 2; m++)
#pragma unroll
      for (int n = 0; n < 4; n++) mma_f64(acc.v[m][n][0], acc.v[m][n][1], a[m], b[n]);
  }
}

// Load (or zero) and store this thread's result elements of a band tile.
__device__ __forceinline__ void mma_load(MmaAcc &acc, const double *__restrict__ T) {
  int r0, c0, g, t;
  mma_coords(r0, c0, g, t);
#pragma unroll
  for (int m = 0; m < 2; m++)
#pragma unroll
    for (int n = 0; n < 4; n++)
#pragma unroll
      for (int q = 0; q < 2; q++) acc.v[m][n][q] = T ? T[(r0 + 8 * m + g) * LDT + c0 + 8 * n + 2 * t + q] : 0.0;
}

// T -= acc at this thread's result elements (one subtraction each, after
// the whole product: the order of the reference's blocked update, C - A^T B
// with the product formed first).
__device__ __forceinline__ void mma_sub_store(double *T, const MmaAcc &acc) {
  int r0, c0, g, t;
  mma_coords(r0, c0, g, t);
#pragma unroll
  for (int m = 0; m < 2; m++)
#pragma unroll
    for (int n = 0; n < 4; n++)
#pragma unroll
      for (int q = 0; q < 2; q++) {
        double *c = &T[(r0 + 8 * m + g) * LDT + c0 + 8 * n + 2 * t + q];
        *c = *c - acc.v[m][n][q];
      }
}

__device__ __forceinline__ void mma_store(double *T, const MmaAcc &acc) {
  int r0, c0, g, t;
  mma_coords(r0, c0, g, t);
#pragma unroll
  for (int m = 0; m < 2; m++)
#pragma unroll
    for (int n = 0; n < 4; n++)
#pragma unroll
      for (int q = 0; q < 2; q++) T[(r0 + 8 * m + g) * LDT + c0 + 8 * n + 2 * t + q] = acc.v[m][n][q];
}

// Off-diagonal tiles of block row k: U(k, k+i) = U_kk^-T A(k, k+i), for the
// tiles inside the envelope (i <= jb[k]); the others stay zero.
__global__ void __launch_bounds__(256, 3) k_trsm(const SysDesc *__restrict__ sys, int k) {
  const SysDesc S = sys[blockIdx.y];
  const int i = blockIdx.x + 1;
  if (k >= S.nblk || i > S.J || k + i >= S.nblk || (S.jb && i > S.jb[k])) return;
  extern __shared__ __align__(16) double smt[];
  double *X = smt, *B = X + NB * LDM;
  double *T = S.tiles + ((size_t)(k + i) * (S.J + 1) + i) * TSZ;
  tile_stage_mma(X, S.dinv + (size_t)k * TSZ);
  tile_stage_mma(B, T);
  cp_async_commit();
  MmaAcc acc;
  mma_load(acc, nullptr);
  cp_async_wait_all();
  __syncthreads();
  mma_tn(acc, X, B, false);
  mma_store(T, acc);
}

// Trailing update inside the band: A(k+i, k+j) -= U(k,k+i)^T U(k,k+j),
// 1 <= i <= j <= jb[k] (every other product has a zero factor).  The product is formed in the accumulators from zero and
// subtracted from the target tile once: accumulating into the target
// instead moved an ill-conditioned mode's solution 170 times further from
// LAPACK's (1.3e-12 -> 2.2e-10 relative, config 5's pressure mode 1).
__global__ void __launch_bounds__(256, 3) k_update(const SysDesc *__restrict__ sys, int k,
                                                   const int2 *__restrict__ pairs) {
  const SysDesc S = sys[blockIdx.y];
  const int2 pr = pairs[blockIdx.x];
  const int i = pr.x, j = pr.y;
  if (k >= S.nblk || j > S.J || k + j >= S.nblk || (S.jb && j > S.jb[k])) return;
  extern __shared__ __align__(16) double smt[];
  double *A = smt, *B = A + NB * LDM;
  const size_t J1 = S.J + 1;
  double *Ct = S.tiles + ((size_t)(k + j) * J1 + (j - i)) * TSZ;
  tile_stage_mma(A, S.tiles + ((size_t)(k + i) * J1 + i) * TSZ);
  tile_stage_mma(B, S.tiles + ((size_t)(k + j) * J1 + j) * TSZ);
  cp_async_commit();
  MmaAcc acc;
  mma_load(acc, nullptr);
  cp_async_wait_all();
  __syncthreads();
  mma_tn(acc, A, B, false);
  mma_sub_store(Ct, acc);
}

// ---------------------------------------------------------------------------
// Jacobi diagonal (JACPCG)
// ---------------------------------------------------------------------------

// Element::HelmholtzDiag (src/element.cpp:1512-1561), emap order.
__global__ void k_elem_diag(MeshView M, double hCon, double *__restrict__ ediag) {
  const int e = blockIdx.x, np = M.np, nn = M.npnp;
  const size_t eo = (size_t)e * nn;
  const bool q3 = M.hasQ3[e];
  for (int a = threadIdx.x; a < nn; a += blockDim.x) {
    const int ij = M.emap[a], i = ij / np, j = ij - i * np;
    double s = 0.0;
    for (int q = 0; q < np; q++) s += M.Q1[eo + i * np + q] * (M.D[q * np + j] * M.D[q * np + j]);
    double dg = s;
    s = 0.0;
    for (int p = 0; p < np; p++) s += M.Q2[eo + p * np + j] * (M.D[p * np + i] * M.D[p * np + i]);
    dg += s;
    if (q3) dg += 2.0 * M.Q3[eo + ij] * M.D[j * np + j] * M.D[i * np + i];
    dg += hCon * M.Q4[eo + ij];
    ediag[eo + a] = dg;
  }
}

// PC[g] = 1 / (mixed terms + sum of element diagonals) for boundary nodes,
// 1 / element diagonal for interior nodes (src/matrix.cpp:290-310).
__global__ void k_diag_dss(MeshView M, const double *__restrict__ ediag, double *pc, float *pcf) {
  const int npts = M.nglobal + M.nel * M.nint;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= npts) return;
  double s = 0.0;
  if (g < M.nglobal) {
    for (int q = M.nat_ptr[g]; q < M.nat_ptr[g + 1]; q++) {
      const int bi = M.nat_idx[q], b = bi / M.np, i = bi - b * M.np;
      if (M.b_kind[b] == SX_BC_MIXED) s += M.b_K[b] * M.b_area[bi];
    }
    for (int q = M.g2e_ptr[g]; q < M.g2e_ptr[g + 1]; q++) {
      const int ei = M.g2e_idx[q], e = ei / M.next, i = ei - e * M.next;
      s += ediag[(size_t)e * M.npnp + i];
    }
  } else {
    const int r = g - M.nglobal, e = r / M.nint, i = r - e * M.nint;
    s = ediag[(size_t)e * M.npnp + M.next + i];
  }
  pc[g] = 1.0 / s;
  pcf[g] = (float)(1.0 / s);
}

// ---------------------------------------------------------------------------
// Host drivers
// ---------------------------------------------------------------------------

static int check_status(DBuf<int> &st) {
  int h = 0;
  SX_CUDA(cudaMemcpy(&h, st.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (h & (1 << SX_ERR_SINGULAR_HII)) {
    set_error("interior matrix hii is singular");
    return SX_ERR_SINGULAR_HII;
  }
  if (h & (1 << SX_ERR_BAND)) {
    set_error("btog couples nodes further apart than nband - 1");
    return SX_ERR_BAND;
  }
  if (h & (1 << SX_ERR_NOT_SPD)) {
    set_error("failed to factor Helmholtz matrix (not positive definite)");
    return SX_ERR_NOT_SPD;
  }
  return SX_OK;
}

size_t System::bytes() const {
  return (tiles.n + dinv.n + hbi.n + hii.n + pc.n) * 8 + (hbif.n + hiif.n + pcf.n) * 4;
}

int system_check_status(System &S) { return S.status.p ? check_status(S.status) : SX_OK; }

int factor_batch(std::vector<System *> &systems, cudaStream_t st, bool sync) {
  if (systems.empty()) return SX_OK;
  std::vector<SysDesc> hd(systems.size());
  int maxblk = 0, maxJ = 0;
  for (size_t s = 0; s < systems.size(); s++) {
    System &S = *systems[s];
    const sx_mesh_s &Mh = *S.mesh;
    hd[s] = SysDesc{S.tiles.p, S.dinv.p, S.nblk, S.J, S.status.p, Mh.denv.p + Mh.env_nblk};
    maxblk = std::max(maxblk, S.nblk);
    maxJ = std::max(maxJ, S.J);
  }
  // tiles of block row k over the systems (the launches' extent)
  std::vector<int> rowmax(std::max(maxblk, 1), 0);
  for (System *Sp : systems) {
    const sx_mesh_s &Mh = *Sp->mesh;
    for (int k = 0; k < Sp->nblk; k++)
      rowmax[k] = std::max(rowmax[k], std::min(std::min(Sp->J, Mh.env[Mh.env_nblk + k]), Sp->nblk - 1 - k));
  }
  DBuf<SysDesc> dd;
  SX_TRY(dd.upload_on(hd.data(), hd.size(), st));
  std::vector<int2> pairs;
  for (int j = 1; j <= maxJ; j++)
    for (int i = 1; i <= j; i++) pairs.push_back(make_int2(i, j));
  DBuf<int2> dpairs;
  if (!pairs.empty()) SX_TRY(dpairs.upload_on(pairs.data(), pairs.size(), st));
  const size_t smm = 2 * NB * LDM * sizeof(double), sm2 = 2 * TSZ * sizeof(double);
  SX_CUDA(cudaFuncSetAttribute(k_potrf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
  SX_CUDA(cudaFuncSetAttribute(k_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smm));
  SX_CUDA(cudaFuncSetAttribute(k_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smm));
  const int ns = (int)systems.size();
  for (int k = 0; k < maxblk; k++) {
    k_potrf<<<ns, 256, sm2, st>>>(dd.p, k);
    const int m = rowmax[k];
    if (m > 0) {
      // pairs are listed by j, so those with j <= m come first
      k_trsm<<<dim3(m, ns), 256, smm, st>>>(dd.p, k);
      k_update<<<dim3((unsigned)(m * (m + 1) / 2), ns), 256, smm, st>>>(dd.p, k, dpairs.p);
    }
  }
  SX_CUDA(cudaGetLastError());
  if (sync) SX_CUDA(cudaStreamSynchronize(st));
  return SX_OK;
}

int system_build_direct(System &S, cudaStream_t st, bool sync) {
  sx_mesh_s &Mh = *S.mesh;
  const MeshView M = Mh.view();
  const double hCon = S.betak2 + S.lambda2;
  S.singular = (S.lambda2 + S.betak2) < EPSSP && (Mh.nglobal - Mh.nsolve) == 0 && !Mh.mixed;
  S.nsolve = S.singular ? Mh.nsolve - 1 : Mh.nsolve;
  const int kd = Mh.nband - 1;
  S.nblk = (S.nsolve + NB - 1) / NB;
  S.J = (kd + NB - 1) / NB;
  if (S.status.p == nullptr) SX_TRY(S.status.alloc_in(1, S.pool, st));
  SX_TRY(S.status.zero(st));
  SX_TRY(S.hbi.alloc_in((size_t)Mh.nel * Mh.next * Mh.nint, S.pool, st));
  SX_TRY(S.hii.alloc_in((size_t)Mh.nel * Mh.nint * Mh.nint, S.pool, st));
  DBuf<double> hbb;
  SX_TRY(hbb.alloc_in((size_t)Mh.nel * Mh.next * Mh.next, S.pool, st, true));
  const size_t smem = condense_smem(M);
  // the kernel's shared-memory limit is a per-function setting: set it once,
  // for the largest order, so that builds of different orders on other host
  // threads never lower it under this launch
  static std::once_flag attr_once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(attr_once, []() {
    attr_err = cudaFuncSetAttribute(k_elem_condense, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)condense_smem_np(NP_MAX));
  });
  SX_CUDA(attr_err);
  k_elem_condense<<<Mh.nel, 256, smem, st>>>(M, hCon, S.hbi.p, S.hii.p, hbb.p, S.status.p);
  SX_CUDA(cudaGetLastError());
  const size_t ntiles = (size_t)std::max(S.nblk, 1) * (S.J + 1);
  SX_TRY(S.tiles.alloc_in(ntiles * TSZ, S.pool, st));
  SX_TRY(S.tiles.zero(st));
  SX_TRY(S.dinv.alloc_in((size_t)std::max(S.nblk, 1) * TSZ, S.pool, st));
  SX_TRY(S.dinv.zero(st));
  if (S.nsolve > 0) {
    const int npad = S.nblk * NB - S.nsolve;
    if (npad > 0) k_band_identity_pad<<<(npad + 127) / 128, 128, 0, st>>>(S.tiles.p, S.J, S.nsolve, S.nblk);
    for (size_t c = 0; c + 1 < Mh.colour_ptr.size(); c++) {
      const int n = Mh.colour_ptr[c + 1] - Mh.colour_ptr[c];
      if (n > 0)
        k_band_add<<<n, 256, 0, st>>>(M, Mh.dcolour_elmt.p + Mh.colour_ptr[c], hbb.p, S.tiles.p, S.J,
                                      S.nsolve, S.status.p);
    }
    if (Mh.mixed) k_band_mixed<<<1, 1, 0, st>>>(M, S.tiles.p, S.J, S.nsolve);
    SX_CUDA(cudaGetLastError());
  }
  if (!sync) return SX_OK;
  SX_CUDA(cudaStreamSynchronize(st));
  SX_TRY(check_status(S.status));
  return SX_OK;
}

int system_build_jacobi(System &S, cudaStream_t st, bool sync) {
  sx_mesh_s &Mh = *S.mesh;
  S.singular = (S.lambda2 + S.betak2) < EPSSP && (Mh.nglobal - Mh.nsolve) == 0 && !Mh.mixed;
  S.nsolve = S.singular ? Mh.nsolve - 1 : Mh.nsolve;
  return system_build_jacobi_diag(S, st, sync);
}

// Inverse Jacobi diagonal only (also used by DIRECT systems for the
// mixed-precision form).
int system_build_jacobi_diag(System &S, cudaStream_t st, bool sync) {
  sx_mesh_s &Mh = *S.mesh;
  const MeshView M = Mh.view();
  const double hCon = S.betak2 + S.lambda2;
  const int npts = Mh.nglobal + Mh.nel * Mh.nint;
  DBuf<double> ediag;
  SX_TRY(ediag.alloc_in((size_t)Mh.nel * Mh.npnp, S.pool, st, true));
  SX_TRY(S.pc.alloc_in(npts, S.pool, st));
  SX_TRY(S.pcf.alloc_in(npts, S.pool, st));
  k_elem_diag<<<Mh.nel, 128, 0, st>>>(M, hCon, ediag.p);
  k_diag_dss<<<(npts + 255) / 256, 256, 0, st>>>(M, ediag.p, S.pc.p, S.pcf.p);
  SX_CUDA(cudaGetLastError());
  if (sync) SX_CUDA(cudaStreamSynchronize(st));
  return SX_OK;
}

// Copy the factor out of the tiles into LAPACK "U" band storage, ldab = nband.
int system_band_export(const System &S, double *ab) {
  const sx_mesh_s &Mh = *S.mesh;
  const int nband = Mh.nband, kd = nband - 1;
  std::vector<double> t((size_t)S.tiles.n);
  SX_CUDA(cudaMemcpy(t.data(), S.tiles.p, t.size() * 8, cudaMemcpyDeviceToHost));
  std::memset(ab, 0, sizeof(double) * (size_t)S.nsolve * nband);
  for (int n = 0; n < S.nsolve; n++)
    for (int m = std::max(0, n - kd); m <= n; m++) ab[(size_t)n * nband + kd + m - n] = t[tile_addr(m, n, S.J)];
  return SX_OK;
}

}  // namespace sx
