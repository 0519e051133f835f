// sx_pcg.cu -- Jacobi-PCG solve on the GPU (Field::solve JACPCG branch,
// src/field.cpp:627-720; Barrett et al. Fig. 2.5).
//
// Vectors are globally numbered (element-boundary globals first, then the
// interior nodes element by element, src/field.cpp:643-647).  The operator
// (Field::HelmholtzOperator, src/field.cpp:771-856) is applied per element
// with the sum-factorised kernel, written to an element-local buffer, and
// summed into the global vector in a fixed element order through the CSR
// inverse of btog: deterministic, no atomics.  Dot products reduce in a
// fixed order (per-block partials, then one block).
#include <cmath>

#include "sx_kernels.cuh"
#include "sx_pcg.cuh"

namespace sx {

constexpr int RED_BLOCKS = 296;  // 2 x 148 SMs
enum { S_R2 = 0, S_RHO1, S_RHO2, S_DOTP, S_ALPHA, S_BETA, S_EPS, S_COUNT };

int PcgWork::reserve(const MeshView &M) {
  const int n = M.nglobal + M.nel * M.nint;
  if (n <= npts) return SX_OK;
  SX_TRY(r.alloc(n));
  SX_TRY(p.alloc(n));
  SX_TRY(q.alloc(n));
  SX_TRY(x.alloc(n));
  SX_TRY(Ye.alloc((size_t)M.nel * M.npnp));
  SX_TRY(part.alloc(RED_BLOCKS));
  SX_TRY(scal.alloc(16));
  npts = n;
  return SX_OK;
}

__device__ __forceinline__ double block_sum(double v, double *sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += sh[i];
  return t;
}

// partial sums of a.b (or a.(w*a) when w != nullptr)
__global__ void __launch_bounds__(256) k_dot(const double *__restrict__ a, const double *__restrict__ b,
                                             const double *__restrict__ w, int n, double *part) {
  __shared__ double sh[8];
  double s = 0.0;
  for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256)
    s += w ? a[i] * (w[i] * a[i]) : a[i] * b[i];
  const double t = block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// Final reduction + scalar recurrence.  mode 0: r2 (and rho2 <- rho1),
// 1: rho1 and beta, 2: dotp and alpha, 3: epsb2 = (tol ||b||)^2.
__global__ void k_dot_final(const double *part, int np, double *scal, int mode, double tol) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) s += part[i];
  // fixed-order tree over the 32 lanes of each warp, then over warps
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x) return;
  double t = 0.0;
  for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += sh[i];
  switch (mode) {
    case 0:
      scal[S_R2] = t;
      scal[S_RHO2] = scal[S_RHO1];
      break;
    case 1:
      scal[S_RHO1] = t;
      scal[S_BETA] = t / scal[S_RHO2];
      break;
    case 2:
      scal[S_DOTP] = t;
      scal[S_ALPHA] = scal[S_RHO1] / t;
      break;
    default: {
      const double e = tol * sqrt(t);
      scal[S_EPS] = e * e;
      scal[S_R2] = 0.0;
    }
  }
}

__global__ void k_pcg_p(const double *__restrict__ pc, const double *__restrict__ r, double *p, int n,
                        const double *scal, int first) {
  const double beta = first ? 0.0 : scal[S_BETA];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double z = pc[i] * r[i];
    p[i] = first ? z : beta * p[i] + z;
  }
}

__global__ void __launch_bounds__(256) k_pcg_xr(double *x, double *r, const double *__restrict__ p,
                                                const double *__restrict__ q, int n, const double *scal,
                                                double *part) {
  __shared__ double sh[8];
  const double alpha = scal[S_ALPHA];
  double s = 0.0;
  for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
    x[i] += alpha * p[i];
    const double rv = r[i] + (-alpha) * q[i];
    r[i] = rv;
    s += rv * rv;
  }
  const double t = block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_zero_range(double *v, int lo, int hi) {
  const int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i < hi) v[i] = 0.0;
}

__global__ void k_sub(double *r, const double *p, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) r[i] -= p[i];
}

// Element half of the operator: Ye[e] = A_e (gathered x), in emap order.
template <int NP>
__global__ void __launch_bounds__(128) k_op_elem(MeshView M, double hCon, const double *__restrict__ x,
                                                 double *__restrict__ Ye) {
  constexpr int NN = NP * NP, NE = 4 * (NP - 1), NI = NN - NE;
  const int e = blockIdx.x, tid = threadIdx.x;
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
  for (int a = tid; a < NN; a += 128) {
    const double v = (a < NE) ? x[M.btog[(size_t)e * NE + a]] : x[M.nglobal + (size_t)e * NI + (a - NE)];
    u[emap[a]] = v;
  }
  __syncthreads();
  helm_op<NP, double>(D, Q[0], Q[1], Q[2], Q[3], M.hasQ3[e] != 0, hCon, u, R, S, out, 128);
  for (int a = tid; a < NN; a += 128) Ye[eo + a] = out[emap[a]];
}

// Assembly half: y[g] = mixed terms (boundary order) + element sums
// (element order); interior copied.  `bc` non-null switches the boundary
// terms to the natural-BC forcing <h, w> (buildRHS) instead of K x.
__global__ void k_op_dss(MeshView M, const double *__restrict__ Ye, const double *__restrict__ x,
                         const double *__restrict__ bc, int rhs_mode, double *y) {
  const int npts = M.nglobal + M.nel * M.nint;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= npts) return;
  if (g < M.nglobal) {
    double s = 0.0;
    if (!rhs_mode && M.mixed)
      for (int q = M.nat_ptr[g]; q < M.nat_ptr[g + 1]; q++) {
        const int bi = M.nat_idx[q], b = bi / M.np;
        if (M.b_kind[b] == SX_BC_MIXED) s += M.b_K[b] * M.b_area[bi] * x[g];
      }
    for (int q = M.g2e_ptr[g]; q < M.g2e_ptr[g + 1]; q++) {
      const int ei = M.g2e_idx[q], e = ei / M.next, i = ei - e * M.next;
      s += Ye[(size_t)e * M.npnp + i];
    }
    if (rhs_mode)
      for (int q = M.nat_ptr[g]; q < M.nat_ptr[g + 1]; q++) {
        const int bi = M.nat_idx[q], b = bi / M.np;
        if (M.b_kind[b] == SX_BC_NATURAL)
          s += (bc ? bc[bi] : 0.0) * M.b_area[bi];
        else
          s += (M.b_K[b] * M.b_C[b]) * M.b_area[bi];
      }
    y[g] = s;
  } else {
    const int r = g - M.nglobal, e = r / M.nint, i = r - e * M.nint;
    y[g] = Ye[(size_t)e * M.npnp + M.next + i];
  }
}

// constrain (src/field.cpp:728-768): Ye[e] = -(M f + H g) in emap order.
template <int NP>
__global__ void __launch_bounds__(128) k_constrain(MeshView M, double hCon, const double *__restrict__ f,
                                                   const double *__restrict__ gess, double *__restrict__ Ye) {
  constexpr int NN = NP * NP, NE = 4 * (NP - 1);
  const int e = blockIdx.x, tid = threadIdx.x;
  __shared__ double D[NN], Q[4][NN], u[NN], R[NN], S[NN], out[NN], F[NN];
  __shared__ int emap[NN];
  const size_t eo = (size_t)e * NN;
  for (int i = tid; i < NN; i += 128) {
    D[i] = M.D[i];
    Q[0][i] = M.Q1[eo + i];
    Q[1][i] = M.Q2[eo + i];
    Q[2][i] = M.Q3[eo + i];
    Q[3][i] = M.Q4[eo + i];
    emap[i] = M.emap[i];
    F[i] = f[eo + i] * M.Q8[eo + i];
    u[i] = 0.0;
  }
  __syncthreads();
  if (M.emask[e]) {
    for (int a = tid; a < NE; a += 128) u[emap[a]] = gess[M.btog[(size_t)e * NE + a]];
    __syncthreads();
    helm_op<NP, double>(D, Q[0], Q[1], Q[2], Q[3], M.hasQ3[e] != 0, hCon, u, R, S, out, 128);
    for (int i = tid; i < NN; i += 128) F[i] += out[i];
    __syncthreads();
  }
  for (int a = tid; a < NN; a += 128) Ye[eo + a] = -F[emap[a]];
}

// local2global of the initial guess (last element wins, as the reference's
// sequential loop, src/field.cpp:928-948); interior copied.
__global__ void k_l2g(MeshView M, const double *__restrict__ u, double *x) {
  const int npts = M.nglobal + M.nel * M.nint;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= npts) return;
  if (g < M.nglobal) {
    const int ei = M.g2e_last[g];
    if (ei < 0) {
      x[g] = 0.0;
      return;
    }
    const int e = ei / M.next, i = ei - e * M.next;
    x[g] = u[(size_t)e * M.npnp + M.emap[i]];
  } else {
    const int r = g - M.nglobal, e = r / M.nint, i = r - e * M.nint;
    x[g] = u[(size_t)e * M.npnp + M.emap[M.next + i]];
  }
}

// global2local + setEssential (src/field.cpp:710-713, 1022-1040).
__global__ void k_g2l(MeshView M, const double *__restrict__ x, const double *__restrict__ gess, double *u) {
  const int e = blockIdx.x;
  const size_t eo = (size_t)e * M.npnp;
  for (int a = threadIdx.x; a < M.npnp; a += blockDim.x) {
    double v;
    if (a < M.next) {
      const int g = M.btog[(size_t)e * M.next + a];
      v = (M.emask[e] && M.bmask[(size_t)e * M.next + a]) ? gess[g] : x[g];
    } else {
      v = x[M.nglobal + (size_t)e * M.nint + (a - M.next)];
    }
    u[eo + M.emap[a]] = v;
  }
}

__global__ void k_essential_one(MeshView M, const double *__restrict__ bc, double *g) {
  if (threadIdx.x || blockIdx.x) return;
  const int np = M.np, nm = np - 1;
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

#define SX_NP_SWITCH(np, CALL)                                                                  \
  switch (np) {                                                                                  \
    case 3: { constexpr int N_ = 3; CALL; } break;                                              \
    case 4: { constexpr int N_ = 4; CALL; } break;                                              \
    case 5: { constexpr int N_ = 5; CALL; } break;                                              \
    case 6: { constexpr int N_ = 6; CALL; } break;                                              \
    case 7: { constexpr int N_ = 7; CALL; } break;                                              \
    case 8: { constexpr int N_ = 8; CALL; } break;                                              \
    case 9: { constexpr int N_ = 9; CALL; } break;                                              \
    case 10: { constexpr int N_ = 10; CALL; } break;                                            \
    case 11: { constexpr int N_ = 11; CALL; } break;                                            \
    case 12: { constexpr int N_ = 12; CALL; } break;                                            \
    default: break;                                                                              \
  }

int global_op(const MeshView &M, double hCon, const double *x, double *y, double *Ye, cudaStream_t st) {
  SX_NP_SWITCH(M.np, (k_op_elem<N_><<<M.nel, 128, 0, st>>>(M, hCon, x, Ye)));
  const int npts = M.nglobal + M.nel * M.nint;
  k_op_dss<<<(npts + 255) / 256, 256, 0, st>>>(M, Ye, x, nullptr, 0, y);
  SX_CUDA(cudaGetLastError());
  return SX_OK;
}

int pcg_solve_job(const MeshView &M, const System &S, PcgWork &W, const Job &job, double tol_rel,
                  int step_max, cudaStream_t st, int *iters_max, double *rel_res, int *launches) {
  SX_TRY(W.reserve(M));
  const int npts = M.nglobal + M.nel * M.nint;
  const int nsolve = S.nsolve, nzero = M.nglobal - nsolve;
  const double hCon = S.betak2 + S.lambda2;
  const int vb = (npts + 255) / 256;
  const int gb = std::min(vb, RED_BLOCKS);
  int rc = SX_OK;
  *iters_max = 0;
  *rel_res = 0.0;
  double *sc = W.scal.p;
  for (int p = 0; p < job.P; p++) {
    double *u = job.u + (size_t)p * job.ustride;
    const double *f = job.f + (size_t)p * job.fstride;
    const double *bc = job.bc ? job.bc + (size_t)p * job.bcstride : nullptr;
    double *g = job.gess + (size_t)p * M.nglobal;
    SX_CUDA(cudaMemsetAsync(g, 0, sizeof(double) * M.nglobal, st));
    if (bc) k_essential_one<<<1, 1, 0, st>>>(M, bc, g);
    SX_CUDA(cudaMemsetAsync(sc, 0, sizeof(double) * 16, st));
    // RHS
    SX_NP_SWITCH(M.np, (k_constrain<N_><<<M.nel, 128, 0, st>>>(M, hCon, f, g, W.Ye.p)));
    k_op_dss<<<vb, 256, 0, st>>>(M, W.Ye.p, nullptr, bc, 1, W.r.p);
    if (nzero > 0) k_zero_range<<<(nzero + 255) / 256, 256, 0, st>>>(W.r.p, nsolve, M.nglobal);
    k_dot<<<gb, 256, 0, st>>>(W.r.p, W.r.p, nullptr, npts, W.part.p);
    k_dot_final<<<1, 256, 0, st>>>(W.part.p, gb, sc, 3, tol_rel);
    // initial residual r = b - A x
    k_l2g<<<vb, 256, 0, st>>>(M, u, W.x.p);
    if (nzero > 0) k_zero_range<<<(nzero + 255) / 256, 256, 0, st>>>(W.x.p, nsolve, M.nglobal);
    SX_TRY(global_op(M, hCon, W.x.p, W.p.p, W.Ye.p, st));
    if (nzero > 0) k_zero_range<<<(nzero + 255) / 256, 256, 0, st>>>(W.p.p, nsolve, M.nglobal);
    k_sub<<<gb, 256, 0, st>>>(W.r.p, W.p.p, npts);
    k_dot<<<gb, 256, 0, st>>>(W.r.p, W.r.p, nullptr, npts, W.part.p);
    k_dot_final<<<1, 256, 0, st>>>(W.part.p, gb, sc, 0, 0.0);
    double hs[8];
    SX_CUDA(cudaMemcpyAsync(hs, sc, sizeof(double) * 8, cudaMemcpyDeviceToHost, st));
    SX_CUDA(cudaStreamSynchronize(st));
    const double epsb2 = hs[S_EPS];
    double r2 = hs[S_R2];
    int i = 0;
    while (r2 > epsb2 && ++i < step_max) {
      k_dot<<<gb, 256, 0, st>>>(W.r.p, nullptr, S.pc.p, npts, W.part.p);
      k_dot_final<<<1, 256, 0, st>>>(W.part.p, gb, sc, 1, 0.0);
      k_pcg_p<<<gb, 256, 0, st>>>(S.pc.p, W.r.p, W.p.p, npts, sc, i == 1);
      SX_TRY(global_op(M, hCon, W.p.p, W.q.p, W.Ye.p, st));
      if (nzero > 0) k_zero_range<<<(nzero + 255) / 256, 256, 0, st>>>(W.q.p, nsolve, M.nglobal);
      k_dot<<<gb, 256, 0, st>>>(W.p.p, W.q.p, nullptr, npts, W.part.p);
      k_dot_final<<<1, 256, 0, st>>>(W.part.p, gb, sc, 2, 0.0);
      k_pcg_xr<<<gb, 256, 0, st>>>(W.x.p, W.r.p, W.p.p, W.q.p, npts, sc, W.part.p);
      k_dot_final<<<1, 256, 0, st>>>(W.part.p, gb, sc, 0, 0.0);
      SX_CUDA(cudaMemcpyAsync(hs, sc, sizeof(double) * 8, cudaMemcpyDeviceToHost, st));
      SX_CUDA(cudaStreamSynchronize(st));
      r2 = hs[S_R2];
    }
    if (i == step_max) rc = SX_WARN_STEP_LIMIT;
    // kernels enqueued for this plane: RHS + initial residual (10, + 3 range
    // zeroings when there are essential nodes, + 1 for BC values), 9 (+1)
    // per iteration body, 1 to unpack
    if (launches) {
      const int zr = nzero > 0 ? 1 : 0;
      const int bodies = (i == step_max) ? i - 1 : i;
      *launches += 10 + 3 * zr + (bc ? 1 : 0) + bodies * (9 + zr) + 1;
    }
    k_g2l<<<M.nel, 128, 0, st>>>(M, W.x.p, g, u);
    SX_CUDA(cudaGetLastError());
    *iters_max = std::max(*iters_max, i);
    const double b2 = epsb2 / (tol_rel * tol_rel);
    if (b2 > 0) *rel_res = std::max(*rel_res, std::sqrt(r2 / b2));
  }
  return rc;
}

}  // namespace sx
