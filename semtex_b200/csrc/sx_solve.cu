// sx_solve.cu -- GPU DIRECT solve of Helmholtz planes (Field::solve, DIRECT
// branch, src/field.cpp:588-624).
//
// A "job" is a set of P planes that share one system (the Re and Im planes
// of a Fourier mode).  Every kernel takes an array of jobs (grid.y = job), so
// the plain form launches one job per mode and the batched form all modes
// at once.  Per job:
//   k_essential   getEssential: essential BC values into a global vector
//                 (src/field.cpp:994-1019, Essential::set src/condition.cpp:80-101)
//   k_rhs_elem    constrain  f <- -(M f + H g)  (src/field.cpp:728-768) and the
//                 element half of local2globalSumSC: edge-major gather,
//                 F_b -= (hbi hii^-1) F_i  (src/element.cpp:356-395)
//   k_rhs_dss     direct-stiffness sum of F_b into the global RHS in element
//                 order, then <h, w> natural/mixed terms in boundary order, then
//                 the essential tail zeroed (src/field.cpp:892-924)
//   band sweeps   U^T y = b, U x = y: LAPACK dpbtrs "U" (src/field.cpp:609),
//                 one thread-block cluster per job (sx_band.cu)
//   k_backsub     global2localSC: u_i = hii^-1 F_i - (hii^-1 h_ib) u_b
//                 (src/element.cpp:398-438), then setEssential
//                 (src/field.cpp:1022-1040)
#include "sx_internal.h"
#include "sx_kernels.cuh"
#include "sx_solve.cuh"

namespace sx {

// ---------------------------------------------------------------------------
// Essential BC values
// ---------------------------------------------------------------------------

// One thread per plane; boundaries in order so later boundaries overwrite
// shared corner nodes exactly as the reference's sequential loop does.
__global__ void k_essential(MeshView M, const Job *__restrict__ jobs) {
  const Job J = jobs[blockIdx.y];
  const int p = threadIdx.x;
  if (p >= J.P || J.bc == nullptr) return;
  const double *bc = J.bc + (size_t)p * J.bcstride;
  double *g = J.gess + (size_t)p * M.nglobal;
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

// ---------------------------------------------------------------------------
// Element forcing and condensation
// ---------------------------------------------------------------------------

template <int NP>
__global__ void __launch_bounds__(128) k_rhs_elem(MeshView M, const Job *__restrict__ jobs) {
  constexpr int NN = NP * NP, NE = 4 * (NP - 1), NI = NN - NE;
  const Job J = jobs[blockIdx.y];
  const int e = blockIdx.x, tid = threadIdx.x;
  __shared__ double D[NN], Q[5][NN], u[NN], R[NN], S[NN], F[NN], Fe[NN];
  __shared__ double hb[NE * (NI > 0 ? NI : 1)];
  __shared__ int emap[NN];
  const size_t eo = (size_t)e * NN;
  for (int i = tid; i < NN; i += 128) {
    D[i] = M.D[i];
    Q[0][i] = M.Q1[eo + i];
    Q[1][i] = M.Q2[eo + i];
    Q[2][i] = M.Q3[eo + i];
    Q[3][i] = M.Q4[eo + i];
    Q[4][i] = M.Q8[eo + i];
    emap[i] = M.emap[i];
  }
  const double *hbi = J.hbi + (size_t)e * NE * NI;
  for (int i = tid; i < NE * NI; i += 128) hb[i] = hbi[i];
  const bool q3 = M.hasQ3[e], masked = M.emask[e] != 0;
  const int *bt = M.btog + (size_t)e * NE;
  __syncthreads();
  for (int p = 0; p < J.P; p++) {
    double *f = J.f + (size_t)p * J.fstride + eo;
    for (int i = tid; i < NN; i += 128) F[i] = Q[4][i] * f[i];
    if (masked) {
      const double *g = J.gess + (size_t)p * M.nglobal;
      for (int i = tid; i < NN; i += 128) u[i] = 0.0;
      __syncthreads();
      for (int i = tid; i < NE; i += 128) u[emap[i]] = g[bt[i]];
      __syncthreads();
      helm_op<NP, double>(D, Q[0], Q[1], Q[2], Q[3], q3, J.hCon, u, R, S, Fe, 128);
      for (int i = tid; i < NN; i += 128) F[i] += Fe[i];
    }
    __syncthreads();
    for (int a = tid; a < NN; a += 128) Fe[a] = -F[emap[a]];
    __syncthreads();
    double *fb = J.Fb + ((size_t)p * M.nel + e) * NE;
    for (int b = tid; b < NE; b += 128) {
      double s = 0.0;
#pragma unroll 7
      for (int q = 0; q < NI; q++) s += hb[b * NI + q] * Fe[NE + q];
      const double v = Fe[b] - s;
      fb[b] = v;
      f[b] = v;
    }
    for (int i = NE + tid; i < NN; i += 128) f[i] = Fe[i];
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Direct-stiffness sum into the condensed RHS
// ---------------------------------------------------------------------------

__global__ void k_rhs_dss(MeshView M, const Job *__restrict__ jobs) {
  const Job J = jobs[blockIdx.y];
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= J.npad) return;
  for (int p = 0; p < J.P; p++) {
    double s = 0.0;
    if (g < J.nsolve) {
      const double *fb = J.Fb + (size_t)p * M.nel * M.next;
      for (int q = M.g2e_ptr[g]; q < M.g2e_ptr[g + 1]; q++) s += fb[M.g2e_idx[q]];
      if (M.nat_ptr[g] < M.nat_ptr[g + 1]) {
        const double *bc = J.bc ? J.bc + (size_t)p * J.bcstride : nullptr;
        for (int q = M.nat_ptr[g]; q < M.nat_ptr[g + 1]; q++) {
          const int bi = M.nat_idx[q], b = bi / M.np;
          if (M.b_kind[b] == SX_BC_NATURAL)
            s += (bc ? bc[bi] : 0.0) * M.b_area[bi];
          else
            s += (M.b_K[b] * M.b_C[b]) * M.b_area[bi];
        }
      }
    }
    J.rhs[(size_t)p * J.rhs_stride + g] = s;
  }
}

// ---------------------------------------------------------------------------
// Interior back-substitution + essential values
// ---------------------------------------------------------------------------

template <int NP>
__global__ void __launch_bounds__(128) k_backsub(MeshView M, const Job *__restrict__ jobs) {
  constexpr int NN = NP * NP, NE = 4 * (NP - 1), NI = NN - NE;
  const Job J = jobs[blockIdx.y];
  const int e = blockIdx.x, tid = threadIdx.x;
  extern __shared__ __align__(16) double smk[];
  double *hii = smk, *hb = hii + NI * NI;
  __shared__ double ub[NE], fi[NI > 0 ? NI : 1];
  __shared__ int emap[NN], bt[NE], bm[NE];
  const double *gi = J.hii + (size_t)e * NI * NI;
  for (int i = tid; i < NI * NI; i += 128) hii[i] = gi[i];
  const double *gb = J.hbi + (size_t)e * NE * NI;
  for (int i = tid; i < NE * NI; i += 128) hb[i] = gb[i];
  for (int i = tid; i < NN; i += 128) emap[i] = M.emap[i];
  for (int i = tid; i < NE; i += 128) {
    bt[i] = M.btog[(size_t)e * NE + i];
    bm[i] = M.bmask[(size_t)e * NE + i];
  }
  const bool masked = M.emask[e] != 0;
  const size_t eo = (size_t)e * NN;
  __syncthreads();
  for (int p = 0; p < J.P; p++) {
    const double *rhs = J.rhs + (size_t)p * J.rhs_stride;
    const double *f = J.f + (size_t)p * J.fstride + eo;
    double *u = J.u + (size_t)p * J.ustride + eo;
    for (int b = tid; b < NE; b += 128) ub[b] = (bt[b] < J.nsolve) ? rhs[bt[b]] : 0.0;
    for (int i = tid; i < NI; i += 128) fi[i] = f[NE + i];
    __syncthreads();
    for (int b = tid; b < NE; b += 128) u[emap[b]] = ub[b];
    for (int r = tid; r < NI; r += 128) {
      double s = 0.0;
      for (int c = 0; c < NI; c++) s += hii[r * NI + c] * fi[c];
      double t = 0.0;
      for (int b = 0; b < NE; b++) t += hb[b * NI + r] * ub[b];
      u[emap[NE + r]] = s - t;
    }
    if (masked) {
      const double *g = J.gess + (size_t)p * M.nglobal;
      for (int b = tid; b < NE; b += 128)
        if (bm[b]) u[emap[b]] = g[bt[b]];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------

template <int NP>
static void launch_elem(const MeshView &M, const Job *djobs, int njobs, bool rhs, cudaStream_t st) {
  constexpr int NN = NP * NP, NE = 4 * (NP - 1), NI = NN - NE;
  dim3 grid(M.nel, njobs);
  if (rhs) {
    k_rhs_elem<NP><<<grid, 128, 0, st>>>(M, djobs);
  } else {
    const size_t sm = sizeof(double) * (NI * NI + NE * NI);
    k_backsub<NP><<<grid, 128, sm, st>>>(M, djobs);
  }
}

template <int NP>
static int prepare_np() {
  constexpr int NN = NP * NP, NE = 4 * (NP - 1), NI = NN - NE;
  const size_t sm = sizeof(double) * (NI * NI + NE * NI);
  SX_CUDA(cudaFuncSetAttribute(k_backsub<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  return SX_OK;
}

static void dispatch_elem(const MeshView &M, const Job *djobs, int njobs, bool rhs, cudaStream_t st) {
  switch (M.np) {
#define SX_CASE(n) \
  case n: launch_elem<n>(M, djobs, njobs, rhs, st); break;
    SX_CASE(3) SX_CASE(4) SX_CASE(5) SX_CASE(6) SX_CASE(7) SX_CASE(8) SX_CASE(9) SX_CASE(10)
    SX_CASE(11) SX_CASE(12)
#undef SX_CASE
    default: break;
  }
}

int prepare_direct_kernels(const MeshView &M) {
  switch (M.np) {
#define SX_CASE(n) \
  case n: SX_TRY(prepare_np<n>()); break;
    SX_CASE(3) SX_CASE(4) SX_CASE(5) SX_CASE(6) SX_CASE(7) SX_CASE(8) SX_CASE(9) SX_CASE(10)
    SX_CASE(11) SX_CASE(12)
#undef SX_CASE
    default: return SX_ERR_UNSUPPORTED;
  }
  return prepare_band_kernels();
}

int direct_rhs_jobs(const MeshView &M, const Job *djobs, const std::vector<Job> &hjobs, cudaStream_t st,
                    int *launches) {
  const int nj = (int)hjobs.size();
  int maxpad = 0;
  bool any_bc = false;
  for (const Job &j : hjobs) {
    maxpad = std::max(maxpad, j.npad);
    any_bc |= j.bc != nullptr;
    SX_CUDA(cudaMemsetAsync(j.gess, 0, sizeof(double) * (size_t)j.P * M.nglobal, st));
  }
  if (any_bc) k_essential<<<dim3(1, nj), 32, 0, st>>>(M, djobs);
  dispatch_elem(M, djobs, nj, true, st);
  k_rhs_dss<<<dim3((maxpad + 255) / 256, nj), 256, 0, st>>>(M, djobs);
  SX_CUDA(cudaGetLastError());
  if (launches) *launches += (any_bc ? 1 : 0) + 2;
  return SX_OK;
}

int direct_backsub_jobs(const MeshView &M, const Job *djobs, int nj, cudaStream_t st, int *launches) {
  dispatch_elem(M, djobs, nj, false, st);
  SX_CUDA(cudaGetLastError());
  if (launches) *launches += 1;
  return SX_OK;
}

int direct_solve_jobs(const MeshView &M, const Job *djobs, const std::vector<Job> &hjobs,
                      cudaStream_t st, int C, int *launches, int stages) {
  int nl = 0;
  SX_TRY(direct_rhs_jobs(M, djobs, hjobs, st, &nl));
  SX_TRY(band_sweep_jobs(djobs, hjobs, C, st, stages));
  SX_TRY(direct_backsub_jobs(M, djobs, (int)hjobs.size(), st, &nl));
  if (launches) *launches = nl + 1;
  return SX_OK;
}

}  // namespace sx
