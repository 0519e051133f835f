// sx_mixed.cu -- mixed-precision batched Helmholtz solve.
//
// Same discrete system as Field::solve (src/field.cpp:509-725), solved for
// every plane of every mode at once by iterative refinement:
//
//   b      = FP64 RHS of the JACPCG branch (constrain + buildRHS,
//            src/field.cpp:641-650), essential tail zero
//   repeat   d  = FP32 Jacobi-PCG on  A d = r  (n_inner iterations of
//                 src/field.cpp:672-704 with FP32 vectors and operator)
//            x += d              (FP64)
//            r  = b - A x        (FP64 operator, FP64 residual)
//   until  ||r|| <= tol ||b|| for every plane
//
// Layout: the FP64 vectors (b, x, the residual) are plane-interleaved,
// V[g * PP + p] (node g, plane p), so a gather or scatter through btog moves
// 32 consecutive planes of one node in one coalesced access; the FP32 CG
// vectors are element vectors (sx_mixed.cuh: CgVecs).  Thread mapping
// everywhere: lane = plane within a chunk of 32 (blockIdx.y = chunk); the
// element kernels give each of their np warps one tensor row and one
// tensor column, the node kernels one node row per warp.
//
// One inner iteration is one kernel, k_cg: the Chronopoulos-Gear form of
// PCG (one global reduction per iteration), element by element --
//   gather w = A u of the previous launch (direct-stiffness sum over the
//   node's holders, in element order), the updates of the element's copies
//   of s, r, p, d, u = PC r, the element operator A_e u_e, and the two dots
//   (r, u) (each node once, by its owner) and (A u, u) = sum_e u_e . A_e u_e.
// Reductions are deterministic trees over the blocks (chunk_sum); the last
// block forms the next iteration's scalars.  Each refinement round is one
// captured CUDA graph; the host reads the residual norms between rounds.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <mutex>

#include "sx_kernels.cuh"
#include "sx_mixed.cuh"
#include "sx_ptx.cuh"
#include "sx_solve.cuh"

namespace sx {

constexpr int MX_ROWS = 8;  // node rows per 256-thread block

__device__ __forceinline__ int gidx(const MeshView &M, int e, int a) {
  return a < M.next ? M.btog[(size_t)e * M.next + a] : M.nglobal + e * M.nint + (a - M.next);
}

__device__ __forceinline__ bool real_plane(const MxParams &P, int p) { return P.active[p] != 0; }

// Direct-stiffness sum of element-local boundary values at global node g,
// in element order (the CSR order): up to four loads issued together.
template <typename T>
__device__ __forceinline__ T dss_gather(const MeshView &M, const T *__restrict__ Y, int g, int PP, int p) {
  const int4 q = M.g2e4[g];
  if (q.w == -2) {
    T s = 0;
    for (int k = M.g2e_ptr[g]; k < M.g2e_ptr[g + 1]; k++) s += Y[(size_t)M.g2e_idx[k] * PP + p];
    return s;
  }
  const T v0 = Y[(size_t)q.x * PP + p];
  const T v1 = q.y >= 0 ? Y[(size_t)q.y * PP + p] : T(0);
  const T v2 = q.z >= 0 ? Y[(size_t)q.z * PP + p] : T(0);
  const T v3 = q.w >= 0 ? Y[(size_t)q.w * PP + p] : T(0);
  return ((v0 + v1) + v2) + v3;
}

// FP64 element results: boundary slots as an element-local buffer
// [nel][next][PP] (gathered through btog's CSR), then interior nodes in
// global order [nel*nint][PP].
__device__ __forceinline__ size_t ye_index(const MeshView &M, int e, int a, int PP) {
  return a < M.next ? ((size_t)e * M.next + a) * PP
                    : ((size_t)M.nel * M.next + (size_t)e * M.nint + (a - M.next)) * PP;
}

// Per-plane sums of (a, b) over the whole grid, deterministic and without
// floating-point atomics, as a two-level tree so that no block sums more
// than a few dozen partials at the end of a launch.  Every block writes its
// total (over its ROWS warps) to part[block]; the last block of each group
// of RED_GROUP blocks (an integer counter per chunk and group) sums the
// group's partials in block order into part[G + group]; the last group to
// finish sums the group totals in group order.  Returns true in warp 0 of
// that last block, with the chunk's totals in fa, fb.  part holds (G +
// ceil(G / RED_GROUP)) * PP double2; cnt holds nch * (1 + ceil(G /
// RED_GROUP)) counters, zero on entry and left zero.
constexpr int RED_GROUP = 32;
inline int red_groups(int G) { return (G + RED_GROUP - 1) / RED_GROUP; }

template <int ROWS>
__device__ __forceinline__ bool chunk_sum(double a, double b, double *part, unsigned *cnt, int blk, int G, int y,
                                          int nch, double &fa, double &fb) {
  __shared__ double sa[ROWS][MX_CH], sb[ROWS][MX_CH];
  __shared__ int last;
  const int row = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = y * MX_CH + lane, PPc = nch * MX_CH;
  const int ngrp = (G + RED_GROUP - 1) / RED_GROUP, grp = blk / RED_GROUP;
  const int g0 = grp * RED_GROUP, gn = min(RED_GROUP, G - g0);
  double2 *P1 = reinterpret_cast<double2 *>(part), *P2 = P1 + (size_t)G * PPc;
  unsigned *cg = cnt + nch + (size_t)y * ngrp;
  // ---- the block's total (warp 0 writes it and alone needs the fence
  // that orders it before the counter)
  sa[row][lane] = a;
  sb[row][lane] = b;
  __syncthreads();
  if (row == 0) {
    double ta = 0.0, tb = 0.0;
    for (int r = 0; r < ROWS; r++) {
      ta += sa[r][lane];
      tb += sb[r][lane];
    }
    P1[(size_t)blk * PPc + p] = make_double2(ta, tb);
    __threadfence();
    if (lane == 0) last = (atomicAdd(&cg[grp], 1u) == (unsigned)gn - 1u);
  }
  __syncthreads();
  if (!last) return false;
  // ---- the group's total, over its blocks in order
  __threadfence();
  double ta = 0.0, tb = 0.0;
  for (int k = row; k < gn; k += ROWS) {
    const double2 v = __ldcg(&P1[(size_t)(g0 + k) * PPc + p]);
    ta += v.x;
    tb += v.y;
  }
  sa[row][lane] = ta;
  sb[row][lane] = tb;
  __syncthreads();
  if (row == 0) {
    ta = tb = 0.0;
    for (int r = 0; r < ROWS; r++) {
      ta += sa[r][lane];
      tb += sb[r][lane];
    }
    P2[(size_t)grp * PPc + p] = make_double2(ta, tb);
    if (lane == 0) cg[grp] = 0;
    __threadfence();
    if (lane == 0) last = (atomicAdd(&cnt[y], 1u) == (unsigned)ngrp - 1u);
  }
  __syncthreads();
  if (!last) return false;
  // ---- the chunk's total, over the groups in order
  __threadfence();
  ta = tb = 0.0;
  for (int k = row; k < ngrp; k += ROWS) {
    const double2 v = __ldcg(&P2[(size_t)k * PPc + p]);
    ta += v.x;
    tb += v.y;
  }
  sa[row][lane] = ta;
  sb[row][lane] = tb;
  __syncthreads();
  if (threadIdx.x == 0) cnt[y] = 0;
  if (row != 0) return false;
  fa = fb = 0.0;
  for (int r = 0; r < ROWS; r++) {
    fa += sa[r][lane];
    fb += sb[r][lane];
  }
  return true;
}

// chunk_sum for the 8-warp node kernels, storing the totals.
__device__ __forceinline__ void chunk_reduce2(double a, double b, double *part, unsigned *cnt, int blk, int G,
                                              int y, int nch, double *outA, double *outB) {
  double fa, fb;
  if (chunk_sum<MX_ROWS>(a, b, part, cnt, blk, G, y, nch, fa, fb)) {
    const int p = y * MX_CH + (threadIdx.x & 31);
    if (outA) outA[p] = fa;
    if (outB) outB[p] = fb;
  }
}

// ---------------------------------------------------------------------------
// tiles of a multi-mesh batch
// ---------------------------------------------------------------------------
//
// A multi-mesh batch launches every kernel once over the tiles of all its
// members of one element order: member m owns tiles [t0[m], t0[m + 1]) of
// the one-dimensional grid (t0[0] = 0, t0[count] = the grid).  A block finds
// its member by counting the prefixes at or below its tile (one ballot per
// 32 members), copies the member's descriptor into shared memory and runs
// the same body as the single-mesh kernel.
struct MxTable {
  const MxMember *mem;
  const int *t0;  // count + 1 tile prefixes
  int count;
};

static_assert(sizeof(MxMember) % 8 == 0, "the descriptor is copied in 8-byte words");

__device__ __forceinline__ bool tile_member(const MxTable &T, MxMember &sB, int &local) {
  __shared__ int sm;
  const int t = blockIdx.x;
  if (threadIdx.x < 32) {
    int c = 0;
    for (int k0 = 1; k0 <= T.count; k0 += 32) {
      const int k = k0 + (int)threadIdx.x;
      c += __popc(__ballot_sync(0xffffffffu, k <= T.count && T.t0[k] <= t));
    }
    if (threadIdx.x == 0) sm = c < T.count ? c : -1;
  }
  __syncthreads();
  const int m = sm;
  if (m < 0) return false;  // block-uniform: past the last tile
  local = t - T.t0[m];
  const unsigned long long *src = reinterpret_cast<const unsigned long long *>(T.mem + m);
  unsigned long long *dst = reinterpret_cast<unsigned long long *>(&sB);
  for (int i = threadIdx.x; i < (int)(sizeof(MxMember) / 8); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  return true;
}

// GLL derivative matrices for np = 3..12, FP32 and FP64, in constant memory:
// the operator indexes them with warp-uniform subscripts (lanes are planes),
// so every read is a constant-cache broadcast and stays off the shared-memory
// pipe.  Filled once per device from the same GLL routine as the mesh.
constexpr int D_TOTAL = 645;  // sum of np^2, np = 3..12
__constant__ float c_Df[D_TOTAL];
__constant__ double c_Dd[D_TOTAL];
template <int NP>
struct DOff {
  static constexpr int v = DOff<NP - 1>::v + (NP - 1) * (NP - 1);
};
template <>
struct DOff<3> {
  static constexpr int v = 0;
};
static int ensure_constD() {
  static std::mutex mu;
  static std::vector<char> done(256, 0);
  int dev = 0;
  SX_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 256 && done[dev]) return SX_OK;
  std::vector<float> f(D_TOTAL);
  std::vector<double> d(D_TOTAL);
  int off = 0;
  for (int np = NP_MIN; np <= NP_MAX; np++) {
    std::vector<double> z, w, D;
    gll_tables(np, z, w, D);
    for (int k = 0; k < np * np; k++) {
      d[off + k] = D[k];
      f[off + k] = (float)D[k];
    }
    off += np * np;
  }
  SX_CUDA(cudaMemcpyToSymbol(c_Df, f.data(), sizeof(float) * D_TOTAL));
  SX_CUDA(cudaMemcpyToSymbol(c_Dd, d.data(), sizeof(double) * D_TOTAL));
  if (dev < 256) done[dev] = 1;
  return SX_OK;
}

// ---------------------------------------------------------------------------
// RHS (FP64)
// ---------------------------------------------------------------------------

// Essential values of plane p into gess (Boundary::set through btog,
// src/boundary.cpp:50-64); one thread per plane.
__device__ __forceinline__ void ess_body(const MxMember &B, int p) {
  const MeshView &M = B.M;
  const MxParams &P = B.P;
  if (threadIdx.x || !P.bc || !real_plane(P, p)) return;
  const int np = M.np, nm = np - 1;
  double *g = P.gess + (size_t)p * M.nglobal;
  const double *bc = P.bc + (size_t)p * P.bcstride;
  for (int b = 0; b < M.nbound; b++) {
    if (M.b_kind[b] != SX_BC_ESSENTIAL) continue;
    const int *bmap = M.btog + (size_t)M.b_elmt[b] * M.next;
    const int side = M.b_side[b];
    const double *src = bc + (size_t)b * np;
    for (int i = 0; i < nm; i++) g[bmap[side * nm + i]] = src[i];
    if (side == 3)
      g[bmap[0]] = src[nm];
    else
      g[bmap[side * nm + nm]] = src[nm];
  }
}

__global__ void k_x_ess(const __grid_constant__ MxMember B) { ess_body(B, blockIdx.x); }

__global__ void k_x_ess_multi(MxTable T) {
  __shared__ MxMember sB;
  int t;
  if (tile_member(T, sB, t)) ess_body(sB, t);
}

// (A_e u)(w, j), j = 0..NP-1, in FP64 for the calling warp's tensor row w
// and lane's plane, on tensor lines as in k_cg: warp w holds row w (the
// x-derivative terms) and column w (the y-derivative terms) in registers,
// the derivative matrix from constant memory with compile-time subscripts.
// u in B0 ([NN][32], tensor order; overwritten on curved elements), B1 an
// exchange buffer; entered with B0 filled and the block synchronised, left
// with both buffers still being read (synchronise before reusing them).
template <int NP>
__device__ __forceinline__ void line_apply64(const MeshView &M, int e, double hc, double *B0, double *B1,
                                             double out[NP]) {
  constexpr int NN = NP * NP, DO = DOff<NP>::v;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t eo = (size_t)e * NN;
  double ur[NP], R[NP], S[NP];
  {
    double uc[NP];
#pragma unroll
    for (int j = 0; j < NP; j++) {
      ur[j] = B0[(w * NP + j) * MX_CH + lane];
      uc[j] = B0[(j * NP + w) * MX_CH + lane];
    }
#pragma unroll
    for (int j = 0; j < NP; j++) {
      double r = 0.0, s = 0.0;
#pragma unroll
      for (int k = 0; k < NP; k++) {
        r += ur[k] * c_Dd[DO + j * NP + k];
        s += c_Dd[DO + j * NP + k] * uc[k];
      }
      R[j] = r;
      S[j] = s;
    }
  }
  if (M.hasQ3[e]) {
    __syncthreads();  // every warp has its u lines: B0 is free
#pragma unroll
    for (int j = 0; j < NP; j++) {
      B1[(w * NP + j) * MX_CH + lane] = R[j];
      B0[(j * NP + w) * MX_CH + lane] = S[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NP; j++) {
      const double s_wj = B0[(w * NP + j) * MX_CH + lane], r_jw = B1[(j * NP + w) * MX_CH + lane];
      R[j] = M.Q1[eo + w * NP + j] * R[j] + M.Q3[eo + w * NP + j] * s_wj;
      S[j] = M.Q2[eo + j * NP + w] * S[j] + M.Q3[eo + j * NP + w] * r_jw;
    }
    __syncthreads();  // B1 is free for the column results
  } else {
#pragma unroll
    for (int j = 0; j < NP; j++) {
      R[j] *= M.Q1[eo + w * NP + j];
      S[j] *= M.Q2[eo + j * NP + w];
    }
  }
#pragma unroll
  for (int i = 0; i < NP; i++) {
    double a = 0.0;
#pragma unroll
    for (int k = 0; k < NP; k++) a += c_Dd[DO + k * NP + i] * S[k];
    B1[(i * NP + w) * MX_CH + lane] = a;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NP; j++) {
    double b = 0.0;
#pragma unroll
    for (int k = 0; k < NP; k++) b += R[k] * c_Dd[DO + k * NP + j];
    const int t = w * NP + j;
    out[j] = M.Q4[eo + t] * ur[j] * hc + B1[t * MX_CH + lane] + b;
  }
}

// Dynamic shared memory of the FP64 element kernels: two [NN][32] buffers
// and the [32][NN | 1] forcing stage.
constexpr size_t x64_smem(int np) {
  return (2 * (size_t)np * np * MX_CH + (size_t)MX_CH * ((np * np) | 1)) * sizeof(double);
}

// Ye at edge-map slot a = -(M f + H g) (Field::constrain), NP warps per
// (element, 32 planes).  The forcing of the 32 planes is staged plane by
// plane with coalesced loads into [32][NN | 1] (an odd row stride keeps the
// lanes' column reads on distinct bank pairs), then read by lane.
template <int NP>
__device__ __forceinline__ void constrain_body(const MxMember &B, int e, int y) {
  constexpr int NN = NP * NP, NE = 4 * (NP - 1), NI = NN - NE, TS = NN | 1;
  const MeshView &M = B.M;
  const MxParams &P = B.P;
  double *__restrict__ Ye = B.Ye;
  extern __shared__ __align__(16) double smx[];
  double *B0 = smx, *B1 = B0 + NN * MX_CH, *T = B1 + NN * MX_CH;
  __shared__ int gtab[NN], emt[NN], tsl[NN];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p0 = y * MX_CH, p = p0 + lane;
  const size_t eo = (size_t)e * NN;
  for (int a = threadIdx.x; a < NN; a += NP * 32) {
    gtab[a] = a < NE ? M.btog[(size_t)e * NE + a] : M.nglobal + e * NI + (a - NE);
    emt[a] = M.emap[a];
    tsl[a] = M.pmap[a];
  }
  for (int i = threadIdx.x; i < MX_CH * NN; i += NP * 32) {
    const int q = i / NN, k = i - q * NN, pl = p0 + q;
    T[q * TS + k] = real_plane(P, pl) ? P.f[(size_t)pl * P.stride + eo + k] : 0.0;
  }
  __syncthreads();
  double F[NP];
#pragma unroll
  for (int j = 0; j < NP; j++) F[j] = M.Q8[eo + w * NP + j] * T[lane * TS + w * NP + j];
  if (M.emask[e]) {  // block-uniform: H g, g the essential values
    const double *g = P.gess + (size_t)p * M.nglobal;
    const bool rp = real_plane(P, p);
#pragma unroll
    for (int k = 0; k < NP; k++) {
      const int a = w + k * NP;
      B0[emt[a] * MX_CH + lane] = (rp && a < NE) ? g[gtab[a]] : 0.0;
    }
    __syncthreads();
    double hg[NP];
    line_apply64<NP>(M, e, P.hcon[p], B0, B1, hg);
#pragma unroll
    for (int j = 0; j < NP; j++) F[j] += hg[j];
  }
#pragma unroll
  for (int j = 0; j < NP; j++) {
    const int t = w * NP + j;
    Ye[ye_index(M, e, tsl[t], P.PP) + p] = -F[j];
  }
}

template <int NP>
__global__ void __launch_bounds__(NP * 32, 2) k_x_constrain(const __grid_constant__ MxMember B) {
  constrain_body<NP>(B, blockIdx.x, blockIdx.y);
}

template <int NP>
__global__ void __launch_bounds__(NP * 32, 2) k_x_constrain_multi(MxTable T) {
  __shared__ MxMember sB;
  int t;
  if (tile_member(T, sB, t)) constrain_body<NP>(sB, t % sB.M.nel, t / sB.M.nel);
}

// b = DSS(Ye) + <h,w>, essential tail zero; x = 0, r = b (FP32); per-plane
// ||b||^2.
__device__ __forceinline__ void rhs_body(const MxMember &B, int blk, int y) {
  const MeshView &M = B.M;
  const MxParams &P = B.P;
  const double *__restrict__ Ye = B.Ye;
  double *b64 = B.b64, *x64 = B.V.x64;
  float *r32 = B.V.r0;
  const int row = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = y * MX_CH + lane, PP = P.PP;
  const int npts = M.nglobal + M.nel * M.nint;
  const int ns = P.nsolve[p];
  const bool rp = real_plane(P, p);
  double bb = 0.0;
  for (int g = blk * MX_ROWS + row; g < npts; g += B.G * MX_ROWS) {
    double s = 0.0;
    if (g < M.nglobal) {
      if (g < ns) {
        s = dss_gather(M, Ye, g, PP, p);
        if (rp)
          for (int q = M.nat_ptr[g]; q < M.nat_ptr[g + 1]; q++) {
            const int bi = M.nat_idx[q], bnd = bi / M.np;
            if (M.b_kind[bnd] == SX_BC_NATURAL)
              s += (P.bc ? P.bc[(size_t)p * P.bcstride + bi] : 0.0) * M.b_area[bi];
            else
              s += (M.b_K[bnd] * M.b_C[bnd]) * M.b_area[bi];
          }
      }
    } else {
      s = Ye[((size_t)M.nel * M.next + (g - M.nglobal)) * PP + p];
    }
    const size_t o = (size_t)g * PP + p;
    b64[o] = s;
    x64[o] = 0.0;
    r32[o] = (float)s;
    bb += s * s;
  }
  chunk_reduce2(bb, 0.0, B.part, B.cnt, blk, B.G, y, B.nch, B.b2, nullptr);
}

__global__ void __launch_bounds__(256) k_x_rhs(const __grid_constant__ MxMember B) {
  rhs_body(B, blockIdx.x, blockIdx.y);
}

__global__ void __launch_bounds__(256) k_x_rhs_multi(MxTable T) {
  __shared__ MxMember sB;
  int t;
  if (tile_member(T, sB, t)) rhs_body(sB, t % sB.G, t / sB.G);
}

// ---------------------------------------------------------------------------
// inner FP32 PCG iteration (Chronopoulos-Gear)
// ---------------------------------------------------------------------------
//
// Chronopoulos & Gear (J. Comput. Appl. Math. 25 (1989) 153-168) carry
// s = A p beside p, so both inner products of an iteration come from the
// same vectors and share one reduction:
//   init  u0 = PC r0, w0 = A u0, gamma0 = (r0,u0), delta0 = (w0,u0),
//         alpha0 = gamma0 / delta0, beta0 = 0
//   it i  p = u + beta p, s = w + beta s, d += alpha p, r -= alpha s,
//         u = PC r, w = A u, gamma' = (r,u), delta = (w,u),
//         beta' = gamma' / gamma, alpha' = gamma' / (delta - beta' gamma' / alpha)
// In exact arithmetic these are the iterates of the Jacobi-PCG loop of
// src/field.cpp:672-704.

enum { CG_INIT = 0, CG_ITER = 1, CG_LAST = 2, CG_MODE = 3 };
// mode flag: read the chunk's stop flag (set when a plane is expected to stop
// well before the round ends; otherwise the read is only latency)
constexpr int CG_CHECK_STOP = 4;

// Element-layout address of (element e, plane chunk y, tensor node t, lane l).
template <int NN>
__device__ __forceinline__ size_t eidx(int e, int nch, int y, int t, int l) {
  return (((size_t)e * nch + y) * NN + t) * MX_CH + l;
}

// Direct-stiffness sum of the element-layout W at global node g, in element
// (CSR) order, from its gather list q (holders packed as element << 8 |
// tensor node; .w == -2: walk the CSR, whose entries are element * next +
// slot, slot -> tensor node through emt).  Every holder of g forms the same
// sum in the same order.
template <int NN>
__device__ __forceinline__ float gather_we(const MeshView &M, const float *__restrict__ W, int4 q, int g, int nch,
                                           int y, int l, const int *emt) {
  if (q.w == -2) {
    float s = 0.0f;
    for (int k = M.g2e_ptr[g]; k < M.g2e_ptr[g + 1]; k++) {
      const int ei = M.g2e_idx[k], eh = ei / M.next;
      s += W[eidx<NN>(eh, nch, y, emt[ei - eh * M.next], l)];
    }
    return s;
  }
  const float v0 = W[eidx<NN>(q.x >> 8, nch, y, q.x & 255, l)];
  const float v1 = q.y >= 0 ? W[eidx<NN>(q.y >> 8, nch, y, q.y & 255, l)] : 0.0f;
  const float v2 = q.z >= 0 ? W[eidx<NN>(q.z >> 8, nch, y, q.z & 255, l)] : 0.0f;
  const float v3 = q.w >= 0 ? W[eidx<NN>(q.w >> 8, nch, y, q.w & 255, l)] : 0.0f;
  return ((v0 + v1) + v2) + v3;
}

// One launch = one iteration for every plane: block (element e, chunk y of
// 32 planes), NP warps.  Thread 0 stages the element's spans of r, s, p, d,
// its own A u and the preconditioner into shared memory with TMA bulk copies
// on one mbarrier while the block loads its tables.  Phase A walks the
// element's nodes in edge-map order (warp w takes slots w, w + NP, ...: the
// boundary slots spread evenly), gathers A u of the previous launch at the
// boundary nodes, updates its copies of s, r, p, d in shared memory and
// writes u = PC r; thread 0 streams the updated spans back with bulk stores
// while the operator runs on tensor lines (warp w owns row w for the
// x-derivative terms and column w for the y-derivative terms, the derivative
// matrix in constant memory with compile-time subscripts); A u is staged in
// shared memory and bulk-stored as well.
// mode CG_INIT: r gathered from the residual's global vector, u = PC r;
//               writes r and A u (W[0]); scalars -> slot 0.
// mode CG_ITER: iteration `it` (W and scalar slots it & 1 in, (it + 1) & 1 out).
// mode CG_LAST: only the owners' d update, folded into x64; no operator.
// Resident blocks per SM that the register budget is set for (shared memory
// allows 3 at np <= 9 and 2 at np <= 11).
constexpr int cg_min_blocks(int np) { return np <= 9 ? 3 : (np <= 11 ? 2 : 1); }
constexpr long long CG_WAIT_LIMIT = CG_WAIT_DEFAULT;  // clock cycles: about a second

// Cycles the first wait for a block's staged spans may take before the
// block records SX_ERR_TIMEOUT; per device, set by sx_set_wait_limit.  The
// block then waits again with CG_WAIT_LIMIT for its copies to land (they
// read valid memory), so it never leaves with copies in flight.
__device__ long long g_cg_wait = CG_WAIT_LIMIT;

int set_cg_wait_limit(long long cycles) {
  SX_CUDA(cudaMemcpyToSymbol(g_cg_wait, &cycles, sizeof(cycles)));
  return SX_OK;
}

// Dynamic shared memory of k_cg: six [NN][32] spans, the [NN][16]
// preconditioner pairs and the element's geometry (one float4 a node).
constexpr size_t cg_smem(int np) { return (size_t)np * np * ((6 * MX_CH + 16) * sizeof(float) + 16); }

template <int NP>
__device__ __forceinline__ void cg_body(const MxMember &B, int e, int y, int it, int mode) {
  constexpr int NN = NP * NP, NE = 4 * (NP - 1), NI = NN - NE, DO = DOff<NP>::v;
  const MeshView &M = B.M;
  const MxParams &P = B.P;
  const CgVecs &V = B.V;
  constexpr uint32_t SPAN = NN * MX_CH * sizeof(float), PSPAN = NN * 16 * sizeof(float);
  // shared spans, NN * 32 floats each: r, s, p, d (updated in place); B1 =
  // the element's own A u, then the column results (and r on curved
  // elements); B0 = u, then s on curved elements, then the A u to store;
  // then the preconditioner pairs [NN][16], then the geometry (Q1..Q4 of
  // each node, staged with the spans so that the operator reads no global
  // memory)
  extern __shared__ __align__(128) float smc[];
  float *Rs = smc, *Ss = Rs + NN * MX_CH, *Ps = Ss + NN * MX_CH, *Ds = Ps + NN * MX_CH;
  float *B1 = Ds + NN * MX_CH, *B0 = B1 + NN * MX_CH, *PCs = B0 + NN * MX_CH;
  float4 *Gs = reinterpret_cast<float4 *>(PCs + NN * 16);
  constexpr uint32_t GSPAN = NN * sizeof(float4);
  __shared__ int gtab[NN], emt[NN];
  __shared__ int4 w4[NE];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int staged;
  const int nch = B.nch, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = y * MX_CH + lane, PP = P.PP;
  const bool check = (mode & CG_CHECK_STOP) != 0;
  mode &= CG_MODE;
  const bool init = mode == CG_INIT, last = mode == CG_LAST;
  // a chunk whose planes have all stopped leaves r, d (and so x) as they
  // are: its blocks skip the iteration (block-uniform, before any barrier);
  // the last one still folds d into x, with alpha = beta = 0
  const bool stopped = check && !init && V.skip[y] != 0;
  if (stopped && !last) return;
  const int cur = init ? 0 : (it & 1), nxt = init ? 0 : (cur ^ 1);
  const bool warm = !init && it > 0;  // s, p, d hold previous iterates
  const size_t base = eidx<NN>(e, nch, y, 0, 0), pbase = ((size_t)e * nch + y) * NN * 16;
  // buffers of this launch, selected without indexing the parameter arrays
  const float *__restrict__ Win = cur ? V.WE[1] : V.WE[0];
  float *__restrict__ Wout = nxt ? V.WE[1] : V.WE[0];
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init_cluster();
    const uint32_t bytes = PSPAN + (last ? 0u : GSPAN) + (init ? 0u : SPAN) + (!init && !last ? SPAN : 0u) +
                           (warm ? (last ? 2u : 3u) * SPAN : 0u);
    mbar_arrive_expect_tx(&bar, bytes);
    bulk_g2s(PCs, V.pcE + pbase, PSPAN, &bar);
    if (!last) bulk_g2s(Gs, M.Gf + (size_t)e * NN, GSPAN, &bar);
    if (!init) bulk_g2s(Rs, V.rE + base, SPAN, &bar);
    if (!init && !last) bulk_g2s(B1, Win + base, SPAN, &bar);
    if (warm) {
      bulk_g2s(Ps, V.pE + base, SPAN, &bar);
      bulk_g2s(Ds, V.dE + base, SPAN, &bar);
      if (!last) bulk_g2s(Ss, V.sE + base, SPAN, &bar);
    }
  }
  for (int a = threadIdx.x; a < NN; a += NP * 32) {
    gtab[a] = a < NE ? M.btog[(size_t)e * NE + a] : M.nglobal + e * NI + (a - NE);
    emt[a] = M.emap[a];
    if (a < NE) w4[a] = M.e2w4[(size_t)e * NE + a];
  }
  const double *gam_in = cur ? V.gam[1] : V.gam[0], *alpha_in = cur ? V.alpha[1] : V.alpha[0];
  const double *beta_in = cur ? V.beta[1] : V.beta[0];
  double *gam_out = nxt ? V.gam[1] : V.gam[0], *alpha_out = nxt ? V.alpha[1] : V.alpha[0];
  double *beta_out = nxt ? V.beta[1] : V.beta[0];
  const int ns = P.nsolve[p];
  float alpha = 0.0f, beta = 0.0f;
  if (!init && !stopped) {
    alpha = (float)alpha_in[p];
    beta = (float)beta_in[p];
  }
  const unsigned long long own = M.owner[e];
  __syncthreads();  // the tables
  // Global loads of phase A -- A u of the previous launch at the element's
  // boundary nodes through their holders (or r at INIT) -- issued now, so
  // that their latency overlaps the staging instead of following it.
  float gv[NP];
#pragma unroll
  for (int k = 0; k < NP; k++) {
    const int a = w + k * NP, g = gtab[a];
    gv[k] = 0.0f;
    if (!(a >= NE || g < ns)) continue;
    if (init)
      gv[k] = V.r0[(size_t)g * PP + p];
    else if (!last && a < NE)
      gv[k] = gather_we<NN>(M, Win, w4[a], g, nch, y, lane, emt);
  }
  // the staged spans: thread 0 waits (bounded) and tells the block; the
  // others then pass the completed phase, which orders the TMA writes for them
  if (threadIdx.x == 0) {
    bool ok = mbar_wait(&bar, 0, g_cg_wait);
    if (!ok) {
      atomicOr(V.status, 1 << SX_ERR_TIMEOUT);
      ok = mbar_wait(&bar, 0, CG_WAIT_LIMIT);  // let the copies land before leaving
    }
    staged = ok;
  }
  __syncthreads();
  if (!staged) return;  // block-uniform
  if (threadIdx.x != 0) mbar_wait(&bar, 0, CG_WAIT_LIMIT);

  // ---- phase A: vector updates at the element's nodes on the staged
  // spans, u = PC r -> B0
  double gam = 0.0;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    const int a = w + k * NP, g = gtab[a], t = emt[a], o = t * MX_CH + lane;
    const bool solve = a >= NE || g < ns;
    const bool mine = a >= NE || ((own >> a) & 1ull);
    const float pc = PCs[t * 16 + (lane >> 1)];
    float un = 0.0f;
    if (init) {
      Rs[o] = gv[k];  // zero at essential nodes
      un = pc * gv[k];
      if (solve && mine) gam += (double)gv[k] * (double)un;
    } else if (solve) {
      const float r = Rs[o];
      const float uo = pc * r;
      const float pp = warm ? uo + beta * Ps[o] : uo;
      const float dd = warm ? Ds[o] + alpha * pp : alpha * pp;
      if (last) {
        if (mine) V.x64[(size_t)g * PP + p] += (double)dd;
      } else {
        const float wv = a >= NE ? B1[o] : gv[k];
        const float s = warm ? wv + beta * Ss[o] : wv;
        const float rn = r - alpha * s;
        un = pc * rn;
        Rs[o] = rn;
        Ss[o] = s;
        Ps[o] = pp;
        Ds[o] = dd;
        if (mine) gam += (double)rn * (double)un;
      }
    }
    if (!last) B0[o] = un;
  }
  if (last) return;  // block-uniform; nothing staged for storing
  // the updated spans go back while the operator runs
  fence_proxy_async_smem();
  __syncthreads();
  if (threadIdx.x == 0) {
    bulk_s2g(V.rE + base, Rs, SPAN);
    if (!init) {
      bulk_s2g(V.sE + base, Ss, SPAN);
      bulk_s2g(V.pE + base, Ps, SPAN);
      bulk_s2g(V.dE + base, Ds, SPAN);
    }
    bulk_commit();
  }

  // ---- operator: out = hc Q4 u + D^T S + R D on tensor lines
  float ur[NP], R[NP], S[NP];
  {
    float uc[NP];
#pragma unroll
    for (int j = 0; j < NP; j++) {
      ur[j] = B0[(w * NP + j) * MX_CH + lane];  // row w
      uc[j] = B0[(j * NP + w) * MX_CH + lane];  // column w
    }
#pragma unroll
    for (int j = 0; j < NP; j++) {
      float r = 0.0f, s = 0.0f;
#pragma unroll
      for (int k = 0; k < NP; k++) {
        r += ur[k] * c_Df[DO + j * NP + k];  // r(w, j) = sum_k u(w, k) D(j, k)
        s += c_Df[DO + j * NP + k] * uc[k];  // s(j, w) = sum_k D(j, k) u(k, w)
      }
      R[j] = r;
      S[j] = s;
    }
  }
  const float4 *G = Gs;
  if (M.hasQ3[e]) {
    // curved: R = Q1 r + Q3 s, S = Q2 s + Q3 r need both at every node
    __syncthreads();  // every warp has its u lines: B0 is free
#pragma unroll
    for (int j = 0; j < NP; j++) {
      B1[(w * NP + j) * MX_CH + lane] = R[j];
      B0[(j * NP + w) * MX_CH + lane] = S[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NP; j++) {
      const float4 gr = G[w * NP + j], gc = G[j * NP + w];
      const float s_wj = B0[(w * NP + j) * MX_CH + lane], r_jw = B1[(j * NP + w) * MX_CH + lane];
      R[j] = gr.x * R[j] + gr.z * s_wj;
      S[j] = gc.y * S[j] + gc.z * r_jw;
    }
    __syncthreads();  // B1 is free for the column results
  } else {
#pragma unroll
    for (int j = 0; j < NP; j++) {
      R[j] *= G[w * NP + j].x;
      S[j] *= G[j * NP + w].y;
    }
  }
  // column w: a(i, w) = sum_k D(k, i) S(k, w), handed to the row owners
#pragma unroll
  for (int i = 0; i < NP; i++) {
    float a = 0.0f;
#pragma unroll
    for (int k = 0; k < NP; k++) a += c_Df[DO + k * NP + i] * S[k];
    B1[(i * NP + w) * MX_CH + lane] = a;
  }
  __syncthreads();
  // row w: out(w, j) = hc Q4 u + a(w, j) + sum_k R(w, k) D(k, j)
  const float hc = (float)P.hcon[p];
  double del = 0.0;
#pragma unroll
  for (int j = 0; j < NP; j++) {
    float b = 0.0f;
#pragma unroll
    for (int k = 0; k < NP; k++) b += R[k] * c_Df[DO + k * NP + j];
    const int t = w * NP + j;
    const float out = G[t].w * hc * ur[j] + B1[t * MX_CH + lane] + b;
    B0[t * MX_CH + lane] = out;  // every warp is past its reads of u in B0
    del += (double)ur[j] * (double)out;
  }
  fence_proxy_async_smem();
  __syncthreads();
  if (threadIdx.x == 0) {
    bulk_s2g(Wout + base, B0, SPAN);
    bulk_commit();
  }

  // ---- gamma = (r, u), delta = (A u, u); the chunk's last block forms the
  // next iteration's scalars
  double gn, dn;
  if (chunk_sum<NP>(gam, del, B.part, B.cnt, e, M.nel, y, nch, gn, dn)) {
    double an, bn;
    if (init) {
      bn = 0.0;
      an = dn > 0.0 ? gn / dn : 0.0;
      V.gam0[p] = gn;
    } else {
      const double go = gam_in[p], ao = alpha_in[p];
      bn = go > 0.0 ? gn / go : 0.0;
      const double den = ao > 0.0 ? dn - bn * gn / ao : dn;
      an = (gn > 0.0 && den > 0.0) ? gn / den : 0.0;
      // a plane whose round has cut (r, PC r) by 1e13 -- about as far as
      // FP32 vectors go -- stops here: alpha = beta = 0 leaves r, d and
      // gamma unchanged, so it stays stopped for the rest of the round
      // (iterating on in FP32 only feeds rounding noise into alpha)
      if (gn <= 1e-13 * V.gam0[p]) an = bn = 0.0;
    }
    if (!isfinite(an) || !isfinite(bn)) an = bn = 0.0;
    gam_out[p] = gn;
    alpha_out[p] = an;
    beta_out[p] = bn;
    const unsigned live = __ballot_sync(0xffffffffu, real_plane(P, p) && (an != 0.0 || bn != 0.0));
    if (lane == 0) V.skip[y] = live == 0u;
  }
  if (threadIdx.x == 0) bulk_wait_read_all();  // the stores have read shared memory
}

template <int NP>
__global__ void __launch_bounds__(NP * 32, cg_min_blocks(NP))
    k_cg(const __grid_constant__ MxMember B, int it, int mode) {
  cg_body<NP>(B, blockIdx.x, blockIdx.y, it, mode);
}

template <int NP>
__global__ void __launch_bounds__(NP * 32, cg_min_blocks(NP)) k_cg_multi(MxTable T, int it, int mode) {
  __shared__ MxMember sB;
  int t;
  if (tile_member(T, sB, t)) cg_body<NP>(sB, t % sB.M.nel, t / sB.M.nel, it, mode);
}

// ---------------------------------------------------------------------------
// FP64 residual
// ---------------------------------------------------------------------------

// Ye = A_e x at the element's slots (FP64), NP warps per (element, 32
// planes): x gathered through btog in slot order, the operator on tensor
// lines (line_apply64).
template <int NP>
__device__ __forceinline__ void op64_body(const MxMember &B, int e, int y) {
  constexpr int NN = NP * NP, NE = 4 * (NP - 1), NI = NN - NE;
  const MeshView &M = B.M;
  const MxParams &P = B.P;
  const double *__restrict__ x64 = B.V.x64;
  double *__restrict__ Ye = B.Ye;
  extern __shared__ __align__(16) double smx[];
  double *B0 = smx, *B1 = B0 + NN * MX_CH;
  __shared__ int gtab[NN], emt[NN], tsl[NN];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = y * MX_CH + lane, PP = P.PP;
  for (int a = threadIdx.x; a < NN; a += NP * 32) {
    gtab[a] = a < NE ? M.btog[(size_t)e * NE + a] : M.nglobal + e * NI + (a - NE);
    emt[a] = M.emap[a];
    tsl[a] = M.pmap[a];
  }
  __syncthreads();
  double xv[NP];
#pragma unroll
  for (int k = 0; k < NP; k++) xv[k] = x64[(size_t)gtab[w + k * NP] * PP + p];
#pragma unroll
  for (int k = 0; k < NP; k++) B0[emt[w + k * NP] * MX_CH + lane] = xv[k];
  __syncthreads();
  double out[NP];
  line_apply64<NP>(M, e, P.hcon[p], B0, B1, out);
#pragma unroll
  for (int j = 0; j < NP; j++) Ye[ye_index(M, e, tsl[w * NP + j], PP) + p] = out[j];
}

template <int NP>
__global__ void __launch_bounds__(NP * 32, 2) k_x_op64(const __grid_constant__ MxMember B) {
  op64_body<NP>(B, blockIdx.x, blockIdx.y);
}

template <int NP>
__global__ void __launch_bounds__(NP * 32, 2) k_x_op64_multi(MxTable T) {
  __shared__ MxMember sB;
  int t;
  if (tile_member(T, sB, t)) op64_body<NP>(sB, t % sB.M.nel, t / sB.M.nel);
}

// r = b - A x (FP64), essential tail zero; the next round's inner solve
// starts from r32 = r (and d = 0, which its first iteration assumes);
// per-plane ||r||^2.
__device__ __forceinline__ void res_body(const MxMember &B, int blk, int y) {
  const MeshView &M = B.M;
  const MxParams &P = B.P;
  const double *__restrict__ Ye = B.Ye;
  const double *__restrict__ b64 = B.b64;
  float *r32 = B.V.r0;
  const int row = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = y * MX_CH + lane, PP = P.PP;
  const int npts = M.nglobal + M.nel * M.nint;
  const int ns = P.nsolve[p];
  double rr = 0.0;
  for (int g = blk * MX_ROWS + row; g < npts; g += B.G * MX_ROWS) {
    double ax = 0.0;
    bool solve = true;
    if (g < M.nglobal) {
      solve = g < ns;
      if (solve) ax = dss_gather(M, Ye, g, PP, p);
    } else {
      ax = Ye[((size_t)M.nel * M.next + (g - M.nglobal)) * PP + p];
    }
    const size_t o = (size_t)g * PP + p;
    const double r = solve ? b64[o] - ax : 0.0;
    r32[o] = (float)r;
    rr += r * r;
  }
  chunk_reduce2(rr, 0.0, B.part, B.cnt, blk, B.G, y, B.nch, B.r2, nullptr);
}

__global__ void __launch_bounds__(256) k_x_res(const __grid_constant__ MxMember B) {
  res_body(B, blockIdx.x, blockIdx.y);
}

__global__ void __launch_bounds__(256) k_x_res_multi(MxTable T) {
  __shared__ MxMember sB;
  int t;
  if (tile_member(T, sB, t)) res_body(sB, t % sB.G, t / sB.G);
}

// u = x at element nodes, essential values from gess (global2local +
// setEssential, src/field.cpp:710-713, 1022-1040); transposed back to the
// caller's plane-major layout through shared memory.
template <int NP>
__device__ __forceinline__ void unpack_body(const MxMember &B, int e, int y) {
  constexpr int NN = NP * NP, NE = 4 * (NP - 1);
  const MeshView &M = B.M;
  const MxParams &P = B.P;
  const double *__restrict__ x64 = B.V.x64;
  // [NN][33]: the store loop reads a column (one plane) across threads, and
  // the odd row length keeps those reads on distinct banks
  constexpr int VS = MX_CH + 1;
  __shared__ double V[NN * VS];
  __shared__ int emap[NN];
  const int tid = threadIdx.x, row = tid >> 5, lane = tid & 31;
  const int p0 = y * MX_CH, p = p0 + lane, PP = P.PP;
  for (int i = tid; i < NN; i += 256) emap[i] = M.emap[i];
  __syncthreads();
  const bool masked = M.emask[e] != 0;
  for (int a = row; a < NN; a += MX_ROWS) {
    double v;
    if (a < NE) {
      const int g = M.btog[(size_t)e * NE + a];
      v = (masked && M.bmask[(size_t)e * NE + a]) ? P.gess[(size_t)p * M.nglobal + g] : x64[(size_t)g * PP + p];
    } else {
      v = x64[((size_t)M.nglobal + (size_t)e * M.nint + (a - NE)) * PP + p];
    }
    V[emap[a] * VS + lane] = v;
  }
  __syncthreads();
  // plane q's NN values are contiguous in the caller's array: all threads
  // over (plane, node) pairs
  for (int i = tid; i < MX_CH * NN; i += 256) {
    const int q = i / NN, k = i - q * NN, pl = p0 + q;
    if (real_plane(P, pl)) P.u[(size_t)pl * P.stride + (size_t)e * NN + k] = V[k * VS + q];
  }
}

template <int NP>
__global__ void __launch_bounds__(256) k_x_unpack(const __grid_constant__ MxMember B) {
  unpack_body<NP>(B, blockIdx.x, blockIdx.y);
}

template <int NP>
__global__ void __launch_bounds__(256) k_x_unpack_multi(MxTable T) {
  __shared__ MxMember sB;
  int t;
  if (tile_member(T, sB, t)) unpack_body<NP>(sB, t % sB.M.nel, t / sB.M.nel);
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------

#define SX_NP_SWITCH_M(np, CALL)                               \
  switch (np) {                                                \
    case 3: { constexpr int N_ = 3; CALL; } break;            \
    case 4: { constexpr int N_ = 4; CALL; } break;            \
    case 5: { constexpr int N_ = 5; CALL; } break;            \
    case 6: { constexpr int N_ = 6; CALL; } break;            \
    case 7: { constexpr int N_ = 7; CALL; } break;            \
    case 8: { constexpr int N_ = 8; CALL; } break;            \
    case 9: { constexpr int N_ = 9; CALL; } break;            \
    case 10: { constexpr int N_ = 10; CALL; } break;          \
    case 11: { constexpr int N_ = 11; CALL; } break;          \
    case 12: { constexpr int N_ = 12; CALL; } break;          \
    default: break;                                            \
  }

static int grid_nodes(int npts) {
  // node-loop kernels: a fixed grid, up to 6 blocks of 8 node rows per SM,
  // each thread taking 4 nodes per pass
  return std::max(1, std::min((npts + 4 * MX_ROWS - 1) / (4 * MX_ROWS), 6 * 148));
}

template <int NP>
static int set_smem_attrs() {
  SX_CUDA(cudaFuncSetAttribute(k_x_constrain<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)x64_smem(NP)));
  SX_CUDA(cudaFuncSetAttribute(k_x_op64<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)x64_smem(NP)));
  SX_CUDA(cudaFuncSetAttribute(k_cg<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cg_smem(NP)));
  // the largest carveout, so that cg_min_blocks(NP) blocks fit an SM
  SX_CUDA(cudaFuncSetAttribute(k_cg<NP>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  return SX_OK;
}

static MxScalPtrs scal_ptrs(const MixedWork &W) {
  double *s = W.scal.p;
  const size_t PP = W.PP;
  MxScalPtrs r;
  r.r2 = s;
  r.b2 = s + PP;
  for (int k = 0; k < 2; k++) {
    r.gam[k] = s + (2 + k) * PP;
    r.alpha[k] = s + (4 + k) * PP;
    r.beta[k] = s + (6 + k) * PP;
  }
  r.gam0 = s + 8 * PP;
  return r;
}

static CgVecs cg_vecs(MixedWork &W) {
  const MxScalPtrs s = scal_ptrs(W);
  CgVecs v;
  v.rE = W.rE.p;
  v.sE = W.sE.p;
  v.pE = W.pE.p;
  v.dE = W.dE.p;
  v.WE[0] = W.WE0.p;
  v.WE[1] = W.WE1.p;
  v.pcE = W.pcE.p;
  v.r0 = W.r0.p;
  v.x64 = W.x64.p;
  v.status = W.status;
  v.skip = W.skip.p;
  for (int k = 0; k < 2; k++) {
    v.gam[k] = s.gam[k];
    v.alpha[k] = s.alpha[k];
    v.beta[k] = s.beta[k];
  }
  v.gam0 = s.gam0;
  return v;
}

// The kernels' descriptor of a solve on mesh M with workspace W (W.prm set).
static MxMember member_of(const MeshView &M, MixedWork &W) {
  const MxScalPtrs s = scal_ptrs(W);
  MxMember B;
  std::memset(&B, 0, sizeof(B));
  B.M = M;
  B.P = W.prm;
  B.V = cg_vecs(W);
  B.Ye = W.Ye64.p;
  B.b64 = W.b64.p;
  B.r2 = s.r2;
  B.b2 = s.b2;
  B.part = W.part.p;
  B.cnt = W.cnt.p;
  B.nch = W.PP / MX_CH;
  B.G = W.G;
  return B;
}

static int enqueue_init(const MeshView &M, MixedWork &W, bool any_bc, cudaStream_t st, int *nl) {
  const MxMember B = member_of(M, W);
  *nl = 0;
  if (any_bc) {
    k_x_ess<<<W.PP, 32, 0, st>>>(B);
    (*nl)++;
  }
  SX_NP_SWITCH_M(M.np, (k_x_constrain<N_><<<dim3(M.nel, B.nch), N_ * 32, x64_smem(N_), st>>>(B)));
  k_x_rhs<<<dim3(W.G, B.nch), 256, 0, st>>>(B);
  *nl += 2;
  SX_CUDA(cudaGetLastError());
  return SX_OK;
}

// One refinement round: the inner solve from r (r0 buffer, d = 0), x += d,
// then the FP64 residual into r0 for the next round.
static int enqueue_round(const MeshView &M, MixedWork &W, int n_inner, bool check_stop, cudaStream_t st,
                         int *nl) {
  const MxMember B = member_of(M, W);
  const dim3 eg(M.nel, B.nch);
  *nl = 0;
  SX_NP_SWITCH_M(M.np, (k_cg<N_><<<eg, N_ * 32, cg_smem(N_), st>>>(B, 0, CG_INIT)));
  for (int it = 0; it < n_inner; it++) {
    const int mode = (it == n_inner - 1 ? CG_LAST : CG_ITER) | (check_stop ? CG_CHECK_STOP : 0);
    SX_NP_SWITCH_M(M.np, (k_cg<N_><<<eg, N_ * 32, cg_smem(N_), st>>>(B, it, mode)));
  }
  SX_NP_SWITCH_M(M.np, (k_x_op64<N_><<<eg, N_ * 32, x64_smem(N_), st>>>(B)));
  k_x_res<<<dim3(W.G, B.nch), 256, 0, st>>>(B);
  *nl = n_inner + 3;
  SX_CUDA(cudaGetLastError());
  return SX_OK;
}

int mixed_profile_iterations(const MeshView &M, MixedWork &W, int reps, cudaStream_t st) {
  // iteration 1 reads what iteration 0 of the last round wrote
  if (W.PP == 0 || W.n_inner < 2 || reps <= 0) return SX_ERR_ARG;
  const MxMember B = member_of(M, W);
  // every chunk works in the timed launches
  SX_CUDA(cudaMemsetAsync(W.skip.p, 0, sizeof(int) * B.nch, st));
  for (int r = 0; r < reps; r++)
    SX_NP_SWITCH_M(M.np, (k_cg<N_><<<dim3(M.nel, B.nch), N_ * 32, cg_smem(N_), st>>>(B, 1, CG_ITER)));
  SX_CUDA(cudaGetLastError());
  return SX_OK;
}

static int capture(cudaStream_t st, cudaGraphExec_t *out, const std::function<int()> &body) {
  cudaGraph_t g = nullptr;
  SX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  const int rc = body();
  const cudaError_t ce = cudaStreamEndCapture(st, &g);
  if (rc != SX_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  SX_CUDA(ce);
  const cudaError_t ie = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  SX_CUDA(ie);
  return SX_OK;
}

// Interleaved preconditioner PCi[g*M + m] from the per-mode systems.
__global__ void k_x_pc(int npts, int M, const float *const *pcs, float *out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= npts) return;
  for (int m = 0; m < M; m++) out[(size_t)g * M + m] = pcs[m][g];
}

// Element-layout preconditioner pairs, pcE[((e * nch + y) * np^2 + t) * 16 +
// q] = the inverse Jacobi diagonal of mode column 16 y + q (clamped to the
// last mode) at the global node of (e, t); lanes 2q and 2q + 1 -- the mode's
// two planes -- read it.
__global__ void k_x_pce(MeshView M, int nch, int Mc, const float *__restrict__ pcf, float *pcE) {
  const int NN = M.npnp;
  const size_t n = (size_t)M.nel * nch * NN * 16;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int q = (int)(i & 15);
    const size_t r = i >> 4;
    const int t = (int)(r % NN);
    const size_t ey = r / NN;
    const int y = (int)(ey % nch), e = (int)(ey / nch);
    const int g = gidx(M, e, M.pmap[t]);
    pcE[i] = pcf[(size_t)g * Mc + min(16 * y + q, Mc - 1)];
  }
}

static int setup(const MeshView &M, MixedWork &W, const std::vector<MxGroup> &groups, int nz, int num_modes,
                 cudaStream_t st) {
  const int npts = M.nglobal + M.nel * M.nint;
  const int PP = ((nz + MX_CH - 1) / MX_CH) * MX_CH;
  const int Mc = std::max(1, num_modes);
  {
    // grow-only: a workspace is reused across solves of different sizes
    auto need = [&](auto &b, size_t n) { return b.n < n ? b.alloc_in(n, W.pool, st) : SX_OK; };
    const size_t n = (size_t)PP * npts;
    W.G = grid_nodes(npts);
    SX_TRY(need(W.b64, n));
    SX_TRY(need(W.x64, n));
    SX_TRY(need(W.Ye64, (size_t)PP * M.nel * M.npnp));
    const size_t ne = (size_t)PP * M.nel * M.npnp;  // one E-vector
    SX_TRY(need(W.r0, n));
    SX_TRY(need(W.rE, ne));
    SX_TRY(need(W.sE, ne));
    SX_TRY(need(W.pE, ne));
    SX_TRY(need(W.dE, ne));
    SX_TRY(need(W.WE0, ne));
    SX_TRY(need(W.WE1, ne));
    SX_TRY(need(W.pcE, ne / 2));
    SX_TRY(need(W.scal, (size_t)MX_NSCAL * PP));
    SX_TRY(need(W.hcon, (size_t)PP));
    SX_TRY(need(W.gess, (size_t)PP * M.nglobal));
    SX_TRY(need(W.nsolve, (size_t)PP));
    SX_TRY(need(W.active, (size_t)PP));
    SX_TRY(need(W.skip, (size_t)PP / MX_CH));
    SX_TRY(need(W.pcf, (size_t)npts * Mc));
    // reduction tree: block and group partials, chunk and group counters
    const int gmax = std::max(W.G, M.nel);
    SX_TRY(need(W.part, (size_t)PP * (gmax + red_groups(gmax)) * 2));
    const size_t ncnt = (size_t)(PP / MX_CH) * (1 + red_groups(gmax));
    if (W.cnt.n < ncnt) {
      SX_TRY(W.cnt.alloc_in(ncnt, W.pool, st));
      SX_TRY(W.cnt.zero(st));
    }
    W.hscal.assign((size_t)2 * PP, 0.0);
    W.PP = PP;
    W.npts = npts;
    W.M = Mc;
  }
  // per-plane constants; planes without a system here (Nyquist, padding,
  // planes of other groups) are inactive and borrow the first group's
  std::vector<double> hc(PP, groups[0].sys->betak2 + groups[0].sys->lambda2);
  std::vector<int> ns(PP, groups[0].sys->nsolve), act(PP, 0);
  std::vector<const float *> pcs(Mc, groups[0].sys->pcf.p);
  for (const MxGroup &g : groups) {
    for (int q = 0; q < g.P; q++) {
      hc[g.plane0 + q] = g.sys->betak2 + g.sys->lambda2;
      ns[g.plane0 + q] = g.sys->nsolve;
      act[g.plane0 + q] = 1;
    }
    if (g.mode < Mc) pcs[g.mode] = g.sys->pcf.p;
  }
  SX_CUDA(cudaMemcpyAsync(W.hcon.p, hc.data(), sizeof(double) * PP, cudaMemcpyHostToDevice, st));
  SX_CUDA(cudaMemcpyAsync(W.nsolve.p, ns.data(), sizeof(int) * PP, cudaMemcpyHostToDevice, st));
  SX_CUDA(cudaMemcpyAsync(W.active.p, act.data(), sizeof(int) * PP, cudaMemcpyHostToDevice, st));
  SX_CUDA(cudaMemsetAsync(W.skip.p, 0, sizeof(int) * (PP / MX_CH), st));
  DBuf<const float *> dp;
  SX_TRY(dp.upload_on(pcs.data(), pcs.size(), st));
  k_x_pc<<<(npts + 255) / 256, 256, 0, st>>>(npts, Mc, dp.p, W.pcf.p);
  const size_t npce = (size_t)M.nel * (PP / MX_CH) * M.npnp * 16;
  k_x_pce<<<(int)std::min<size_t>((npce + 255) / 256, 8 * 148), 256, 0, st>>>(M, PP / MX_CH, Mc, W.pcf.p,
                                                                               W.pcE.p);
  SX_CUDA(cudaGetLastError());
  SX_CUDA(cudaStreamSynchronize(st));
  W.epoch++;
  return SX_OK;
}

static void bind_params(const MeshView &M, MixedWork &W, int nz, double *d_u, double *d_f, const double *d_bc,
                        long long stride) {
  MxParams &P = W.prm;
  P.PP = W.PP;
  P.nz = nz;
  P.active = W.active.p;
  P.M = W.M;
  P.hcon = W.hcon.p;
  P.nsolve = W.nsolve.p;
  P.pcf = W.pcf.p;
  P.f = d_f;
  P.u = d_u;
  P.stride = stride;
  P.bc = d_bc;
  P.bcstride = (long long)std::max(M.nbound, 1) * M.np;
  P.gess = W.gess.p;
}

// Largest relative residual over the planes of one member from its norms
// (r2[0..PP), b2[0..PP)); infinity for a NaN.
static double worst_rel(const double *r2, const double *b2, int PP) {
  double worst = 0.0;
  for (int p = 0; p < PP; p++) {
    const double rel = b2[p] > 0.0 ? std::sqrt(std::max(r2[p], 0.0) / b2[p]) : 0.0;
    if (!(rel == rel)) return INFINITY;
    worst = std::max(worst, rel);
  }
  return worst;
}

int mixed_solve(const MeshView &M, MixedWork &W, const std::vector<MxGroup> &groups, int nz, int num_modes,
                double *d_u, double *d_f, const double *d_bc, long long stride, bool rebuild, double tol_rel,
                int max_refine, int n_inner, bool check_stop, bool graphs, cudaStream_t st,
                sx_solve_stats *stats) {
  if (groups.empty()) return SX_OK;
  if (M.mixed) {
    set_error("mixed-precision form does not take Robin (mixed) boundary conditions");
    return SX_ERR_UNSUPPORTED;
  }
  SX_TRY(ensure_constD());
  if (rebuild || !graphs || !W.g_init || W.n_inner != n_inner || W.graph_epoch != W.epoch ||
      W.check_stop != check_stop) {
    if (W.g_init) cudaGraphExecDestroy(W.g_init);
    if (W.g_round) cudaGraphExecDestroy(W.g_round);
    W.g_init = W.g_round = nullptr;
    SX_TRY(setup(M, W, groups, nz, num_modes, st));
    int attr_rc = SX_OK;
    SX_NP_SWITCH_M(M.np, (attr_rc = set_smem_attrs<N_>()));
    SX_TRY(attr_rc);
    bind_params(M, W, nz, d_u, d_f, d_bc, stride);
    if (graphs) {
      const bool any_bc = d_bc != nullptr;
      SX_TRY(capture(st, &W.g_init, [&]() { return enqueue_init(M, W, any_bc, st, &W.launches_init); }));
      SX_TRY(capture(st, &W.g_round,
                     [&]() { return enqueue_round(M, W, n_inner, check_stop, st, &W.launches_round); }));
    }
    W.n_inner = n_inner;
    W.check_stop = check_stop;
    W.graph_epoch = W.epoch;
  }
  // essential values: zeroed here, set from the BC lines inside g_init
  SX_CUDA(cudaMemsetAsync(W.gess.p, 0, sizeof(double) * (size_t)W.PP * M.nglobal, st));
  if (graphs)
    SX_CUDA(cudaGraphLaunch(W.g_init, st));
  else
    SX_TRY(enqueue_init(M, W, d_bc != nullptr, st, &W.launches_init));
  int rounds = 0, launches = W.launches_init + 1;
  double worst = 0.0;
  const int PP = W.PP;
  for (rounds = 1; rounds <= max_refine; rounds++) {
    if (graphs)
      SX_CUDA(cudaGraphLaunch(W.g_round, st));
    else
      SX_TRY(enqueue_round(M, W, n_inner, check_stop, st, &W.launches_round));
    launches += W.launches_round;
    // r2 and b2 lead the scalar block
    SX_CUDA(cudaMemcpyAsync(W.hscal.data(), W.scal.p, sizeof(double) * 2 * PP, cudaMemcpyDeviceToHost, st));
    SX_CUDA(cudaStreamSynchronize(st));
    worst = worst_rel(W.hscal.data(), W.hscal.data() + PP, PP);
    if (worst <= tol_rel) break;
  }
  if (rounds > max_refine) rounds = max_refine;
  SX_NP_SWITCH_M(M.np, (k_x_unpack<N_><<<dim3(M.nel, PP / MX_CH), 256, 0, st>>>(member_of(M, W))));
  SX_CUDA(cudaGetLastError());
  int solved = 0;
  for (const MxGroup &g : groups) solved += g.P;
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->planes_solved = solved;
    stats->refinements = rounds;
    stats->iterations_max = rounds * n_inner;
    stats->iterations_total = rounds * n_inner * solved;
    stats->final_rel_residual = worst;
    stats->kernel_launches = launches;
  }
  return worst <= tol_rel ? SX_OK : SX_WARN_STEP_LIMIT;
}

// ---------------------------------------------------------------------------
// multi-mesh batch
// ---------------------------------------------------------------------------

void MxBatch::reset() {
  if (g_init) cudaGraphExecDestroy(g_init);
  if (g_round) cudaGraphExecDestroy(g_round);
  g_init = g_round = nullptr;
  cls.clear();
  order.clear();
  noff.clear();
  epochs.clear();
}

MxBatch::~MxBatch() {
  reset();
  for (cudaEvent_t e : events) cudaEventDestroy(e);
  for (cudaStream_t s : streams) cudaStreamDestroy(s);
}

// The three tile tables of class c: element, node and plane tiles.
static MxTable class_table(const MxBatch &B, const MxBatch::Class &c, int kind) {
  MxTable T;
  T.mem = B.mem.p + c.m0;
  T.t0 = B.tiles.p + c.t0 + (size_t)kind * (c.count + 1);
  T.count = c.count;
  return T;
}

// Runs body(c, stream) for every class, each on its own stream, forked from
// and joined back into st (inside a capture this makes parallel branches).
// The class streams and events, created before any capture.
static int ensure_streams(MxBatch &B) {
  const int nc = (int)B.cls.size();
  if (nc < 2) return SX_OK;
  while ((int)B.streams.size() < nc) {
    cudaStream_t s = nullptr;
    SX_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    B.streams.push_back(s);
  }
  while ((int)B.events.size() < nc + 1) {
    cudaEvent_t e = nullptr;
    SX_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    B.events.push_back(e);
  }
  return SX_OK;
}

static int per_class(MxBatch &B, cudaStream_t st,
                     const std::function<int(const MxBatch::Class &, cudaStream_t)> &body) {
  const int nc = (int)B.cls.size();
  if (nc == 1) return body(B.cls[0], st);
  SX_TRY(ensure_streams(B));
  SX_CUDA(cudaEventRecord(B.events[0], st));
  int rc = SX_OK;
  for (int c = 0; c < nc; c++) {
    SX_CUDA(cudaStreamWaitEvent(B.streams[c], B.events[0], 0));
    if (rc == SX_OK) rc = body(B.cls[c], B.streams[c]);
    SX_CUDA(cudaEventRecord(B.events[c + 1], B.streams[c]));
  }
  for (int c = 0; c < nc; c++) SX_CUDA(cudaStreamWaitEvent(st, B.events[c + 1], 0));
  return rc;
}

static int enqueue_init_multi(MxBatch &B, bool any_bc, cudaStream_t st, int *nl) {
  *nl = 0;
  for (auto &c : B.cls) *nl += any_bc ? 3 : 2;
  return per_class(B, st, [&](const MxBatch::Class &c, cudaStream_t s) {
    if (any_bc) k_x_ess_multi<<<c.tp, 32, 0, s>>>(class_table(B, c, 2));
    SX_NP_SWITCH_M(c.np, (k_x_constrain_multi<N_><<<c.te, N_ * 32, x64_smem(N_), s>>>(class_table(B, c, 0))));
    k_x_rhs_multi<<<c.tn, 256, 0, s>>>(class_table(B, c, 1));
    SX_CUDA(cudaGetLastError());
    return SX_OK;
  });
}

static int enqueue_round_multi(MxBatch &B, int n_inner, bool check_stop, cudaStream_t st, int *nl) {
  *nl = (int)B.cls.size() * (n_inner + 3);
  return per_class(B, st, [&](const MxBatch::Class &c, cudaStream_t s) {
    const MxTable Te = class_table(B, c, 0), Tn = class_table(B, c, 1);
    SX_NP_SWITCH_M(c.np, (k_cg_multi<N_><<<c.te, N_ * 32, cg_smem(N_), s>>>(Te, 0, CG_INIT)));
    for (int it = 0; it < n_inner; it++) {
      const int mode = (it == n_inner - 1 ? CG_LAST : CG_ITER) | (check_stop ? CG_CHECK_STOP : 0);
      SX_NP_SWITCH_M(c.np, (k_cg_multi<N_><<<c.te, N_ * 32, cg_smem(N_), s>>>(Te, it, mode)));
    }
    SX_NP_SWITCH_M(c.np, (k_x_op64_multi<N_><<<c.te, N_ * 32, x64_smem(N_), s>>>(Te)));
    k_x_res_multi<<<c.tn, 256, 0, s>>>(Tn);
    SX_CUDA(cudaGetLastError());
    return SX_OK;
  });
}

template <int NP>
static int set_smem_attrs_multi() {
  SX_CUDA(cudaFuncSetAttribute(k_x_constrain_multi<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)x64_smem(NP)));
  SX_CUDA(cudaFuncSetAttribute(k_x_op64_multi<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)x64_smem(NP)));
  SX_CUDA(cudaFuncSetAttribute(k_cg_multi<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cg_smem(NP)));
  SX_CUDA(cudaFuncSetAttribute(k_cg_multi<NP>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  return SX_OK;
}

int mixed_solve_multi(std::vector<MxItem> &items, MxBatch &B, bool rebuild, double tol_rel, int max_refine,
                      int n_inner, bool check_stop, bool graphs, cudaStream_t st) {
  const int n = (int)items.size();
  if (n == 0) return SX_OK;
  for (const MxItem &it : items) {
    if (it.M.mixed) {
      set_error("mixed-precision form does not take Robin (mixed) boundary conditions");
      return SX_ERR_UNSUPPORTED;
    }
    if (it.groups.empty() || !it.W) return SX_ERR_ARG;
  }
  SX_TRY(ensure_constD());
  bool any_bc = false;
  for (const MxItem &it : items) any_bc |= it.bc != nullptr;
  bool stale = (int)B.order.size() != n || B.epochs.size() != B.order.size();
  for (int m = 0; !stale && m < n; m++) stale = items[B.order[m]].W->epoch != B.epochs[m];
  if (rebuild || stale || !graphs || !B.g_init || B.n_inner != n_inner || B.check_stop != check_stop) {
    B.reset();
    // members by element order, then item order
    B.order.resize(n);
    for (int i = 0; i < n; i++) B.order[i] = i;
    std::stable_sort(B.order.begin(), B.order.end(),
                     [&](int a, int b) { return items[a].M.np < items[b].M.np; });
    std::vector<MxMember> mem(n);
    size_t ntot = 0;
    for (int m = 0; m < n; m++) {
      MxItem &it = items[B.order[m]];
      SX_TRY(setup(it.M, *it.W, it.groups, it.nz, it.num_modes, st));
      int attr_rc = SX_OK;
      SX_NP_SWITCH_M(it.M.np, (attr_rc = set_smem_attrs_multi<N_>()));
      SX_TRY(attr_rc);
      bind_params(it.M, *it.W, it.nz, it.u, it.f, it.bc, it.stride);
      B.noff.push_back(ntot);
      ntot += 2 * (size_t)it.W->PP;
    }
    SX_TRY(B.norms.n < ntot ? B.norms.alloc(ntot) : SX_OK);
    B.hnorms.assign(ntot, 0.0);
    std::vector<int> tiles;
    for (int m = 0; m < n; m++) {
      MxItem &it = items[B.order[m]];
      mem[m] = member_of(it.M, *it.W);
      mem[m].r2 = B.norms.p + B.noff[m];
      mem[m].b2 = mem[m].r2 + it.W->PP;
      if (B.cls.empty() || B.cls.back().np != it.M.np) {
        MxBatch::Class c;
        c.np = it.M.np;
        c.m0 = m;
        B.cls.push_back(c);
      }
      B.cls.back().count++;
    }
    for (auto &c : B.cls) {
      c.t0 = tiles.size();
      std::vector<int> te(1, 0), tn(1, 0), tp(1, 0);
      for (int m = c.m0; m < c.m0 + c.count; m++) {
        const MxMember &b = mem[m];
        te.push_back(te.back() + b.M.nel * b.nch);
        tn.push_back(tn.back() + b.G * b.nch);
        tp.push_back(tp.back() + b.P.PP);
      }
      c.te = te.back();
      c.tn = tn.back();
      c.tp = tp.back();
      tiles.insert(tiles.end(), te.begin(), te.end());
      tiles.insert(tiles.end(), tn.begin(), tn.end());
      tiles.insert(tiles.end(), tp.begin(), tp.end());
    }
    B.epochs.clear();
    for (int m = 0; m < n; m++) B.epochs.push_back(items[B.order[m]].W->epoch);
    SX_TRY(B.mem.n < (size_t)n ? B.mem.alloc(n) : SX_OK);
    SX_TRY(B.tiles.n < tiles.size() ? B.tiles.alloc(tiles.size()) : SX_OK);
    SX_CUDA(cudaMemcpyAsync(B.mem.p, mem.data(), sizeof(MxMember) * n, cudaMemcpyHostToDevice, st));
    SX_CUDA(cudaMemcpyAsync(B.tiles.p, tiles.data(), sizeof(int) * tiles.size(), cudaMemcpyHostToDevice, st));
    SX_CUDA(cudaStreamSynchronize(st));
    SX_TRY(ensure_streams(B));
    if (graphs) {
      SX_TRY(capture(st, &B.g_init, [&]() { return enqueue_init_multi(B, any_bc, st, &B.launches_init); }));
      SX_TRY(capture(st, &B.g_round,
                     [&]() { return enqueue_round_multi(B, n_inner, check_stop, st, &B.launches_round); }));
    }
    B.n_inner = n_inner;
    B.check_stop = check_stop;
  }
  // essential values: zeroed here, set from the BC lines inside the init
  for (const MxItem &it : items)
    SX_CUDA(cudaMemsetAsync(it.W->gess.p, 0, sizeof(double) * (size_t)it.W->PP * it.M.nglobal, st));
  if (graphs)
    SX_CUDA(cudaGraphLaunch(B.g_init, st));
  else
    SX_TRY(enqueue_init_multi(B, any_bc, st, &B.launches_init));
  int rounds = 0, launches = B.launches_init + (int)B.cls.size();
  std::vector<double> worst(n, 0.0);
  for (rounds = 1; rounds <= max_refine; rounds++) {
    if (graphs)
      SX_CUDA(cudaGraphLaunch(B.g_round, st));
    else
      SX_TRY(enqueue_round_multi(B, n_inner, check_stop, st, &B.launches_round));
    launches += B.launches_round;
    SX_CUDA(cudaMemcpyAsync(B.hnorms.data(), B.norms.p, sizeof(double) * B.hnorms.size(), cudaMemcpyDeviceToHost,
                            st));
    SX_CUDA(cudaStreamSynchronize(st));
    bool all = true;
    for (int m = 0; m < n; m++) {
      const int PP = items[B.order[m]].W->PP;
      const double *r2 = B.hnorms.data() + B.noff[m];
      worst[m] = worst_rel(r2, r2 + PP, PP);
      all &= worst[m] <= tol_rel;
    }
    if (all) break;
  }
  if (rounds > max_refine) rounds = max_refine;
  SX_TRY(per_class(B, st, [&](const MxBatch::Class &c, cudaStream_t s) {
    SX_NP_SWITCH_M(c.np, (k_x_unpack_multi<N_><<<c.te, 256, 0, s>>>(class_table(B, c, 0))));
    SX_CUDA(cudaGetLastError());
    return SX_OK;
  }));
  int rc = SX_OK;
  for (int m = 0; m < n; m++) {
    MxItem &it = items[B.order[m]];
    int solved = 0;
    for (const MxGroup &g : it.groups) solved += g.P;
    sx_solve_stats &S = it.stats;
    std::memset(&S, 0, sizeof(S));
    S.planes_solved = solved;
    S.refinements = rounds;
    S.iterations_max = rounds * n_inner;
    S.iterations_total = rounds * n_inner * solved;
    S.final_rel_residual = worst[m];
    S.kernel_launches = launches;
    if (!(worst[m] <= tol_rel)) rc = SX_WARN_STEP_LIMIT;
  }
  return rc;
}

}  // namespace sx
