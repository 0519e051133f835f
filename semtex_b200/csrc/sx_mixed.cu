// sx_mixed.cu -- mixed-precision batched Helmholtz solve.
//
// Same discrete system as Field::solve (src/field.cpp:509-725), solved for
// every plane of every mode at once by iterative refinement:
//
//   b      = FP64 RHS of the JACPCG branch (constrain + buildRHS,
//            src/field.cpp:641-650), essential tail zero
//   repeat   d  = FP32 Jacobi-PCG on  A d = r  (n_inner iterations,
//                 src/field.cpp:672-704 with FP32 vectors and operator)
//            x += d              (FP64)
//            r  = b - A x        (FP64 operator, FP64 residual)
//   until  ||r|| <= tol ||b|| for every plane
//
// One inner iteration is two kernels, each with its reduction fused in:
//   k_mx_op32   p <- z + beta p (z = PC r) on the fly, element operator
//               q_e = A_e p_e (FP32 sum factorisation), interior q stored,
//               boundary contributions to an element-local buffer, and
//               p.q = sum_e p_e . q_e (equal to the assembled dot because p
//               vanishes on essential nodes)
//   k_mx_upd    direct-stiffness gather of q (element order), d += alpha p,
//               r -= alpha q, rho = r.(PC r)
// Reductions are two-level and deterministic: per-block partials, the last
// block to finish sums them in index order.  Each refinement round is one
// captured CUDA graph; the host reads the residual norms between rounds.
#include <cmath>
#include <cstring>
#include <functional>

#include "sx_kernels.cuh"
#include "sx_mixed.cuh"
#include "sx_solve.cuh"

namespace sx {

// ---------------------------------------------------------------------------
// deterministic per-plane reduction of a pair of values
// ---------------------------------------------------------------------------

__device__ __forceinline__ void reduce_pair(double a, double b, double *part, unsigned *cnt, int maxblk,
                                            int nblk, int plane, int bid, double *outA, double *outB) {
  __shared__ double sa[32], sb[32];
  __shared__ int last;
  a = warp_sum(a);
  b = warp_sum(b);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (l == 0) {
    sa[w] = a;
    sb[w] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int i = 0; i < nw; i++) {
      ta += sa[i];
      tb += sb[i];
    }
    double *pp = part + ((size_t)plane * maxblk + bid) * 2;
    pp[0] = ta;
    pp[1] = tb;
    __threadfence();
    const unsigned t = atomicAdd(&cnt[plane], 1u);
    last = (t == (unsigned)(nblk - 1));
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  const double *pp = part + (size_t)plane * maxblk * 2;
  double ta = 0.0, tb = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
    ta += __ldcg(&pp[2 * i]);
    tb += __ldcg(&pp[2 * i + 1]);
  }
  ta = warp_sum(ta);
  tb = warp_sum(tb);
  __syncthreads();
  if (l == 0) {
    sa[w] = ta;
    sb[w] = tb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double fa = 0.0, fb = 0.0;
    for (int i = 0; i < nw; i++) {
      fa += sa[i];
      fb += sb[i];
    }
    if (outA) *outA = fa;
    if (outB) *outB = fb;
    cnt[plane] = 0;
  }
}

// global index of local (edge-map order) node a of element e
__device__ __forceinline__ int gidx(const MeshView &M, int e, int a) {
  return a < M.next ? M.btog[(size_t)e * M.next + a] : M.nglobal + e * M.nint + (a - M.next);
}

// ---------------------------------------------------------------------------
// RHS (FP64)
// ---------------------------------------------------------------------------

__global__ void k_mx_ess(MeshView M, const MxPlane *__restrict__ planes) {
  const MxPlane P = planes[blockIdx.x];
  if (threadIdx.x || P.bc == nullptr) return;
  const int np = M.np, nm = np - 1;
  for (int b = 0; b < M.nbound; b++) {
    if (M.b_kind[b] != SX_BC_ESSENTIAL) continue;
    const int *bmap = M.btog + (size_t)M.b_elmt[b] * M.next;
    const int side = M.b_side[b];
    const double *src = P.bc + (size_t)b * np;
    for (int i = 0; i < nm; i++) P.gess[bmap[side * nm + i]] = src[i];
    if (side == 3)
      P.gess[bmap[0]] = src[nm];
    else
      P.gess[bmap[side * nm + nm]] = src[nm];
  }
}

// Ye[plane][e] = -(M f + H g) in edge-map order (Field::constrain).
template <int NP>
__global__ void __launch_bounds__(128) k_mx_constrain(MeshView M, const MxPlane *__restrict__ planes,
                                                      double *__restrict__ Ye) {
  constexpr int NN = NP * NP, NE = 4 * (NP - 1);
  const MxPlane P = planes[blockIdx.y];
  const int e = blockIdx.x, tid = threadIdx.x;
  __shared__ double D[NN], Q[4][NN], u[NN], R[NN], S[NN], out[NN], F[NN];
  __shared__ int emap[NN];
  const size_t eo = (size_t)e * NN;
  for (int i = tid; i < NN; i += 128) {
    D[i] = M.D[i];
    emap[i] = M.emap[i];
    F[i] = P.f[eo + i] * M.Q8[eo + i];
  }
  if (M.emask[e]) {
    for (int i = tid; i < NN; i += 128) {
      Q[0][i] = M.Q1[eo + i];
      Q[1][i] = M.Q2[eo + i];
      Q[2][i] = M.Q3[eo + i];
      Q[3][i] = M.Q4[eo + i];
      u[i] = 0.0;
    }
    __syncthreads();
    for (int a = tid; a < NE; a += 128) u[emap[a]] = P.gess[M.btog[(size_t)e * NE + a]];
    __syncthreads();
    helm_op<NP, double>(D, Q[0], Q[1], Q[2], Q[3], M.hasQ3[e] != 0, P.hCon, u, R, S, out, 128);
    for (int i = tid; i < NN; i += 128) F[i] += out[i];
  }
  __syncthreads();
  double *y = Ye + ((size_t)blockIdx.y * M.nel + e) * NN;
  for (int a = tid; a < NN; a += 128) y[a] = -F[emap[a]];
}

// b = DSS(Ye) + <h,w>, essential tail zero; x = 0, d = 0, r = b (FP32),
// p_0 = PC r; reduces ||b||^2 and rho_0.
__global__ void __launch_bounds__(256) k_mx_rhs(MeshView M, const MxPlane *__restrict__ planes,
                                                const double *__restrict__ Ye, double *b64, double *x64,
                                                float *r32, float *d32, float *p0, MxScal *scal,
                                                double *part, unsigned *cnt, int maxblk) {
  const int plane = blockIdx.y;
  const MxPlane P = planes[plane];
  const int npts = M.nglobal + M.nel * M.nint;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const size_t o = (size_t)plane * npts;
  double bb = 0.0, rz = 0.0;
  if (g < npts) {
    double s = 0.0;
    const double *y = Ye + (size_t)plane * M.nel * M.npnp;
    if (g < M.nglobal) {
      if (g < P.nsolve) {
        for (int q = M.g2e_ptr[g]; q < M.g2e_ptr[g + 1]; q++) {
          const int ei = M.g2e_idx[q], e = ei / M.next, i = ei - e * M.next;
          s += y[(size_t)e * M.npnp + i];
        }
        for (int q = M.nat_ptr[g]; q < M.nat_ptr[g + 1]; q++) {
          const int bi = M.nat_idx[q], bnd = bi / M.np;
          if (M.b_kind[bnd] == SX_BC_NATURAL)
            s += (P.bc ? P.bc[bi] : 0.0) * M.b_area[bi];
          else
            s += (M.b_K[bnd] * M.b_C[bnd]) * M.b_area[bi];
        }
      }
    } else {
      const int r = g - M.nglobal, e = r / M.nint, i = r - e * M.nint;
      s = y[(size_t)e * M.npnp + M.next + i];
    }
    b64[o + g] = s;
    x64[o + g] = 0.0;
    const float rf = (float)s;
    r32[o + g] = rf;
    d32[o + g] = 0.0f;
    const float z = P.pcf[g] * rf;
    p0[o + g] = z;
    bb = s * s;
    rz = (double)rf * (double)z;
  }
  double *ob = &scal[plane].b2;
  reduce_pair(bb, rz, part, cnt, maxblk, gridDim.x, plane, blockIdx.x, ob, &scal[plane].rho[0]);
}

// ---------------------------------------------------------------------------
// inner FP32 PCG iteration
// ---------------------------------------------------------------------------

template <int NP>
__global__ void __launch_bounds__(128) k_mx_op32(MeshView M, const MxPlane *__restrict__ planes,
                                                 const float *__restrict__ r32, const float *__restrict__ pold,
                                                 float *__restrict__ pnew, float *__restrict__ q32,
                                                 float *__restrict__ Yb, MxScal *scal, int it,
                                                 double *part, unsigned *cnt, int maxblk) {
  constexpr int NN = NP * NP, NE = 4 * (NP - 1), NI = NN - NE;
  const int plane = blockIdx.y;
  const MxPlane P = planes[plane];
  const int e = blockIdx.x, tid = threadIdx.x;
  const int npts = M.nglobal + M.nel * M.nint;
  const size_t o = (size_t)plane * npts;
  __shared__ float D[NN], Q[4][NN], u[NN], R[NN], S[NN], out[NN];
  __shared__ int emap[NN];
  const size_t eo = (size_t)e * NN;
  float beta = 0.0f;
  if (it > 0) {
    const double rn = scal[plane].rho[it & 1], ro = scal[plane].rho[(it - 1) & 1];
    beta = (ro != 0.0) ? (float)(rn / ro) : 0.0f;
  }
  for (int i = tid; i < NN; i += 128) {
    D[i] = M.Df[i];
    Q[0][i] = M.Q1f[eo + i];
    Q[1][i] = M.Q2f[eo + i];
    Q[2][i] = M.Q3f[eo + i];
    Q[3][i] = M.Q4f[eo + i];
    emap[i] = M.emap[i];
  }
  __syncthreads();
  for (int a = tid; a < NN; a += 128) {
    const int g = gidx(M, e, a);
    float pv;
    if (it == 0) {
      pv = pold[o + g];
    } else {
      const float z = P.pcf[g] * r32[o + g];
      pv = z + beta * pold[o + g];
      // one writer per global node: the last element that touches it
      if (a >= NE || M.g2e_last[g] == e * NE + a) pnew[o + g] = pv;
    }
    u[emap[a]] = pv;
  }
  __syncthreads();
  helm_op<NP, float>(D, Q[0], Q[1], Q[2], Q[3], M.hasQ3[e] != 0, (float)P.hCon, u, R, S, out, 128);
  double pq = 0.0;
  for (int a = tid; a < NN; a += 128) {
    const float qv = out[emap[a]];
    pq += (double)(u[emap[a]] * qv);
    if (a < NE)
      Yb[((size_t)plane * M.nel + e) * NE + a] = qv;
    else
      q32[o + M.nglobal + (size_t)e * NI + (a - NE)] = qv;
  }
  reduce_pair(pq, 0.0, part, cnt, maxblk, gridDim.x, plane, blockIdx.x, &scal[plane].pq[it & 1], nullptr);
}

__global__ void __launch_bounds__(256) k_mx_upd(MeshView M, const MxPlane *__restrict__ planes,
                                                const float *__restrict__ pcur, const float *__restrict__ q32,
                                                const float *__restrict__ Yb, float *d32, float *r32,
                                                double *x64, MxScal *scal, int it, int last, double *part,
                                                unsigned *cnt, int maxblk) {
  const int plane = blockIdx.y;
  const MxPlane P = planes[plane];
  const int npts = M.nglobal + M.nel * M.nint;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const size_t o = (size_t)plane * npts;
  const double rho = scal[plane].rho[it & 1], pq = scal[plane].pq[it & 1];
  const float alpha = (pq > 0.0) ? (float)(rho / pq) : 0.0f;
  double rz = 0.0;
  if (g < npts) {
    float q = 0.0f;
    if (g < M.nglobal) {
      if (g < P.nsolve) {
        const float *yb = Yb + (size_t)plane * M.nel * M.next;
        for (int k = M.g2e_ptr[g]; k < M.g2e_ptr[g + 1]; k++) q += yb[M.g2e_idx[k]];
      }
    } else {
      q = q32[o + g];
    }
    const float p = pcur[o + g];
    const float d = d32[o + g] + alpha * p;
    const float r = r32[o + g] - alpha * q;
    r32[o + g] = r;
    if (last)
      x64[o + g] += (double)d;
    else
      d32[o + g] = d;
    const float z = P.pcf[g] * r;
    rz = (double)r * (double)z;
  }
  reduce_pair(rz, 0.0, part, cnt, maxblk, gridDim.x, plane, blockIdx.x, &scal[plane].rho[(it + 1) & 1],
              nullptr);
}

// ---------------------------------------------------------------------------
// FP64 residual
// ---------------------------------------------------------------------------

template <int NP>
__global__ void __launch_bounds__(128) k_mx_op64(MeshView M, const MxPlane *__restrict__ planes,
                                                 const double *__restrict__ x64, double *__restrict__ Ye) {
  constexpr int NN = NP * NP;
  const MxPlane P = planes[blockIdx.y];
  const int e = blockIdx.x, tid = threadIdx.x;
  const int npts = M.nglobal + M.nel * M.nint;
  const size_t o = (size_t)blockIdx.y * npts;
  __shared__ double D[NN], Q[4][NN], u[NN], R[NN], S[NN], out[NN];
  __shared__ int emap[NN];
  const size_t eo = (size_t)e * NN;
  for (int i = tid; i < NN; i += 128) {
    D[i] = M.D[i];
    Q[0][i] = M.Q1[eo + i];
    Q[1][i] = M.Q2[eo + i];
    Q[2][i] = M.Q3[eo + i];
    Q[3][i] = M.Q4[eo + i];
    emap[i] = M.emap[i];
  }
  __syncthreads();
  for (int a = tid; a < NN; a += 128) u[emap[a]] = x64[o + gidx(M, e, a)];
  __syncthreads();
  helm_op<NP, double>(D, Q[0], Q[1], Q[2], Q[3], M.hasQ3[e] != 0, P.hCon, u, R, S, out, 128);
  double *y = Ye + ((size_t)blockIdx.y * M.nel + e) * NN;
  for (int a = tid; a < NN; a += 128) y[a] = out[emap[a]];
}

// r = b - A x (FP64), essential tail zero; restart the inner solve:
// r32 = r, d = 0, p_0 = PC r; reduces ||r||^2 and rho_0.
__global__ void __launch_bounds__(256) k_mx_res(MeshView M, const MxPlane *__restrict__ planes,
                                                const double *__restrict__ Ye, const double *__restrict__ b64,
                                                float *r32, float *d32, float *p0, MxScal *scal, double *part,
                                                unsigned *cnt, int maxblk) {
  const int plane = blockIdx.y;
  const MxPlane P = planes[plane];
  const int npts = M.nglobal + M.nel * M.nint;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const size_t o = (size_t)plane * npts;
  double rr = 0.0, rz = 0.0;
  if (g < npts) {
    double ax = 0.0;
    bool solve = true;
    const double *y = Ye + (size_t)plane * M.nel * M.npnp;
    if (g < M.nglobal) {
      solve = g < P.nsolve;
      if (solve)
        for (int q = M.g2e_ptr[g]; q < M.g2e_ptr[g + 1]; q++) {
          const int ei = M.g2e_idx[q], e = ei / M.next, i = ei - e * M.next;
          ax += y[(size_t)e * M.npnp + i];
        }
    } else {
      const int r = g - M.nglobal, e = r / M.nint, i = r - e * M.nint;
      ax = y[(size_t)e * M.npnp + M.next + i];
    }
    const double r = solve ? b64[o + g] - ax : 0.0;
    const float rf = (float)r;
    r32[o + g] = rf;
    d32[o + g] = 0.0f;
    const float z = P.pcf[g] * rf;
    p0[o + g] = z;
    rr = r * r;
    rz = (double)rf * (double)z;
  }
  reduce_pair(rr, rz, part, cnt, maxblk, gridDim.x, plane, blockIdx.x, &scal[plane].r2, &scal[plane].rho[0]);
}

// u = x at element nodes, essential values from gess (global2local +
// setEssential, src/field.cpp:710-713, 1022-1040).
__global__ void k_mx_unpack(MeshView M, const MxPlane *__restrict__ planes, const double *__restrict__ x64) {
  const MxPlane P = planes[blockIdx.y];
  const int e = blockIdx.x;
  const int npts = M.nglobal + M.nel * M.nint;
  const size_t o = (size_t)blockIdx.y * npts, eo = (size_t)e * M.npnp;
  for (int a = threadIdx.x; a < M.npnp; a += blockDim.x) {
    double v;
    if (a < M.next) {
      const int g = M.btog[(size_t)e * M.next + a];
      v = (M.emask[e] && M.bmask[(size_t)e * M.next + a]) ? P.gess[g] : x64[o + g];
    } else {
      v = x64[o + M.nglobal + (size_t)e * M.nint + (a - M.next)];
    }
    P.u[eo + M.emap[a]] = v;
  }
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

static int reserve(const MeshView &M, MixedWork &W, int planes) {
  const int npts = M.nglobal + M.nel * M.nint;
  if (planes <= W.planes && npts == W.npts) return SX_OK;
  const size_t n = (size_t)planes * npts;
  SX_TRY(W.b64.alloc(n));
  SX_TRY(W.x64.alloc(n));
  SX_TRY(W.Ye64.alloc((size_t)planes * M.nel * M.npnp));
  SX_TRY(W.r32.alloc(n));
  SX_TRY(W.d32.alloc(n));
  SX_TRY(W.pA.alloc(n));
  SX_TRY(W.pB.alloc(n));
  SX_TRY(W.q32.alloc(n));
  SX_TRY(W.Yb32.alloc((size_t)planes * M.nel * M.next));
  SX_TRY(W.scal.alloc(planes));
  W.maxblk = std::max(M.nel, (npts + 255) / 256);
  SX_TRY(W.partA.alloc((size_t)planes * W.maxblk * 2));
  SX_TRY(W.cntA.alloc(planes));
  SX_TRY(W.cntA.zero());
  W.hscal.resize(planes);
  W.planes = planes;
  W.npts = npts;
  return SX_OK;
}

static int enqueue_init(const MeshView &M, MixedWork &W, int P, bool any_bc, cudaStream_t st, int *nl) {
  const int npts = W.npts;
  *nl = 0;
  if (any_bc) {
    k_mx_ess<<<P, 32, 0, st>>>(M, W.dplanes.p);
    (*nl)++;
  }
  SX_NP_SWITCH_M(M.np, (k_mx_constrain<N_><<<dim3(M.nel, P), 128, 0, st>>>(M, W.dplanes.p, W.Ye64.p)));
  k_mx_rhs<<<dim3((npts + 255) / 256, P), 256, 0, st>>>(M, W.dplanes.p, W.Ye64.p, W.b64.p, W.x64.p, W.r32.p,
                                                        W.d32.p, W.pA.p, W.scal.p, W.partA.p, W.cntA.p,
                                                        W.maxblk);
  *nl += 2;
  SX_CUDA(cudaGetLastError());
  return SX_OK;
}

static int enqueue_round(const MeshView &M, MixedWork &W, int P, int n_inner, cudaStream_t st, int *nl) {
  const int npts = W.npts;
  *nl = 0;
  for (int it = 0; it < n_inner; it++) {
    float *pold = (it & 1) ? W.pA.p : W.pB.p;  // p_{it-1} lives in buffer (it-1)&1
    float *pcur = (it & 1) ? W.pB.p : W.pA.p;  // p_it in buffer it&1
    if (it == 0) pold = W.pA.p;                // p_0 written by the restart
    SX_NP_SWITCH_M(M.np, (k_mx_op32<N_><<<dim3(M.nel, P), 128, 0, st>>>(
                             M, W.dplanes.p, W.r32.p, pold, pcur, W.q32.p, W.Yb32.p, W.scal.p, it, W.partA.p,
                             W.cntA.p, W.maxblk)));
    k_mx_upd<<<dim3((npts + 255) / 256, P), 256, 0, st>>>(M, W.dplanes.p, pcur, W.q32.p, W.Yb32.p, W.d32.p,
                                                          W.r32.p, W.x64.p, W.scal.p, it,
                                                          it == n_inner - 1 ? 1 : 0, W.partA.p, W.cntA.p,
                                                          W.maxblk);
    *nl += 2;
  }
  SX_NP_SWITCH_M(M.np, (k_mx_op64<N_><<<dim3(M.nel, P), 128, 0, st>>>(M, W.dplanes.p, W.x64.p, W.Ye64.p)));
  k_mx_res<<<dim3((npts + 255) / 256, P), 256, 0, st>>>(M, W.dplanes.p, W.Ye64.p, W.b64.p, W.r32.p, W.d32.p,
                                                        W.pA.p, W.scal.p, W.partA.p, W.cntA.p, W.maxblk);
  *nl += 2;
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

int mixed_solve(const MeshView &M, MixedWork &W, const std::vector<MxPlane> &planes, bool rebuild,
                double tol_rel, int max_refine, int n_inner, cudaStream_t st, sx_solve_stats *stats) {
  const int P = (int)planes.size();
  if (P == 0) return SX_OK;
  if (M.mixed) {
    set_error("mixed-precision form does not take Robin (mixed) boundary conditions");
    return SX_ERR_UNSUPPORTED;
  }
  SX_TRY(reserve(M, W, P));
  bool any_bc = false;
  for (const MxPlane &p : planes) any_bc |= p.bc != nullptr;
  if (rebuild || !W.g_init || W.n_inner != n_inner) {
    if (W.g_init) cudaGraphExecDestroy(W.g_init);
    if (W.g_round) cudaGraphExecDestroy(W.g_round);
    W.g_init = W.g_round = nullptr;
    if (W.dplanes.n < (size_t)P) SX_TRY(W.dplanes.alloc(P));
    SX_CUDA(cudaMemcpy(W.dplanes.p, planes.data(), sizeof(MxPlane) * P, cudaMemcpyHostToDevice));
    SX_TRY(capture(st, &W.g_init, [&]() { return enqueue_init(M, W, P, any_bc, st, &W.launches_init); }));
    SX_TRY(capture(st, &W.g_round, [&]() { return enqueue_round(M, W, P, n_inner, st, &W.launches_round); }));
    W.n_inner = n_inner;
  }
  // essential values: zeroed, then set from the BC lines inside g_init
  for (const MxPlane &p : planes) SX_CUDA(cudaMemsetAsync(p.gess, 0, sizeof(double) * M.nglobal, st));
  SX_CUDA(cudaGraphLaunch(W.g_init, st));
  int rounds = 0, launches = W.launches_init;
  double worst = 0.0;
  for (rounds = 1; rounds <= max_refine; rounds++) {
    SX_CUDA(cudaGraphLaunch(W.g_round, st));
    launches += W.launches_round;
    SX_CUDA(cudaMemcpyAsync(W.hscal.data(), W.scal.p, sizeof(MxScal) * P, cudaMemcpyDeviceToHost, st));
    SX_CUDA(cudaStreamSynchronize(st));
    worst = 0.0;
    for (int i = 0; i < P; i++) {
      const double b2 = W.hscal[i].b2, r2 = W.hscal[i].r2;
      const double rel = b2 > 0.0 ? std::sqrt(std::max(r2, 0.0) / b2) : 0.0;
      if (!(rel == rel)) worst = INFINITY;  // NaN
      worst = std::max(worst, rel);
    }
    if (worst <= tol_rel) break;
  }
  if (rounds > max_refine) rounds = max_refine;
  k_mx_unpack<<<dim3(M.nel, P), 128, 0, st>>>(M, W.dplanes.p, W.x64.p);
  launches += 1;
  SX_CUDA(cudaGetLastError());
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->planes_solved = P;
    stats->refinements = rounds;
    stats->iterations_max = rounds * n_inner;
    stats->iterations_total = rounds * n_inner * P;
    stats->final_rel_residual = worst;
    stats->kernel_launches = launches;
  }
  return worst <= tol_rel ? SX_OK : SX_WARN_STEP_LIMIT;
}

}  // namespace sx
