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

// One block of ELEM_WARPS warps per (element, job); both planes of the job in
// one pass, so the element's hbi block is read once per job.  Warp w owns
// rows b = w, w + ELEM_WARPS, ... of hbi (hbi hii^-1), its lanes the row's
// NI columns: the whole block is loaded into registers, coalesced and
// evict-first (it is not read again before the band sweeps have streamed
// the factor through L2), before anything else, so that it arrives while
// the forcing and the element operator are computed.  The geometric factors
// of the operator are read only for elements that hold essential nodes.
constexpr int ELEM_WARPS = 4;

template <int NP>
__global__ void __launch_bounds__(ELEM_WARPS * 32) k_rhs_elem(MeshView M, const Job *__restrict__ jobs) {
  constexpr int NN = NP * NP, NE = 4 * (NP - 1), NI = NN - NE;
  constexpr int NT = ELEM_WARPS * 32, RW = (NE + ELEM_WARPS - 1) / ELEM_WARPS, QL = (NI + 31) / 32;
  const Job J = jobs[blockIdx.y];
  const int e = blockIdx.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int P = J.P;
  const double *hbi = J.hbi + (size_t)e * NE * NI;
  double h[RW][QL];
#pragma unroll
  for (int k = 0; k < RW; k++)
#pragma unroll
    for (int j = 0; j < QL; j++) {
      const int b = w + ELEM_WARPS * k, q = lane + 32 * j;
      h[k][j] = (b < NE && q < NI) ? __ldcs(hbi + b * NI + q) : 0.0;
    }
  __shared__ double F[2][NN], Fe[2][NN];
  __shared__ double D[NN], Q[4][NN], u[NN], R[NN], S[NN], T[NN];
  __shared__ int emap[NN];
  const size_t eo = (size_t)e * NN;
  const bool masked = M.emask[e] != 0;
  for (int i = tid; i < NN; i += NT) {
    emap[i] = M.emap[i];
    const double q8 = M.Q8[eo + i];
    for (int p = 0; p < P; p++) F[p][i] = q8 * J.f[(size_t)p * J.fstride + eo + i];
  }
  if (masked) {
    // f <- M f + H g: the operator applied to the element's essential values
    for (int i = tid; i < NN; i += NT) {
      D[i] = M.D[i];
      Q[0][i] = M.Q1[eo + i];
      Q[1][i] = M.Q2[eo + i];
      Q[2][i] = M.Q3[eo + i];
      Q[3][i] = M.Q4[eo + i];
    }
    const bool q3 = M.hasQ3[e];
    const int *bt = M.btog + (size_t)e * NE;
    for (int p = 0; p < P; p++) {
      const double *g = J.gess + (size_t)p * M.nglobal;
      __syncthreads();
      for (int i = tid; i < NN; i += NT) u[i] = 0.0;
      __syncthreads();
      for (int i = tid; i < NE; i += NT) u[emap[i]] = g[bt[i]];
      __syncthreads();
      helm_op<NP, double>(D, Q[0], Q[1], Q[2], Q[3], q3, J.hCon, u, R, S, T, NT);
      for (int i = tid; i < NN; i += NT) F[p][i] += T[i];
    }
  }
  __syncthreads();
  // boundary-first element ordering, negated: f <- -(M f + H g)
  for (int a = tid; a < NN; a += NT)
    for (int p = 0; p < P; p++) Fe[p][a] = -F[p][emap[a]];
  __syncthreads();
  // F_b -= (hbi hii^-1) F_i: row b of the block against the interior values
#pragma unroll
  for (int k = 0; k < RW; k++) {
    const int b = w + ELEM_WARPS * k;
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int j = 0; j < QL; j++) {
      const int q = lane + 32 * j;
      if (q < NI) {
        s0 += h[k][j] * Fe[0][NE + q];
        if (P > 1) s1 += h[k][j] * Fe[1][NE + q];
      }
    }
    s0 = warp_sum(s0);
    if (P > 1) s1 = warp_sum(s1);
    if (lane == 0 && b < NE) {
      const double v0 = Fe[0][b] - s0;
      J.Fb[(size_t)e * NE + b] = v0;
      J.f[eo + b] = v0;
      if (P > 1) {
        const double v1 = Fe[1][b] - s1;
        J.Fb[((size_t)M.nel + e) * NE + b] = v1;
        J.f[(size_t)J.fstride + eo + b] = v1;
      }
    }
  }
  for (int i = NE + tid; i < NN; i += NT)
    for (int p = 0; p < P; p++) J.f[(size_t)p * J.fstride + eo + i] = Fe[p][i];
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

// Threads of k_backsub: one per interior row, rounded up to whole warps.
template <int NP>
__host__ __device__ constexpr int back_threads() {
  return ((NP * NP - 4 * (NP - 1) + 31) / 32) * 32;
}

// One block per (element, job), both planes in one pass.  Thread r owns
// interior row r: u_i[r] = sum_c hii^-1[r][c] F_i[c] - sum_b (hbi hii^-1)[b][r] u_b[b].
// hii^-1 is stored column-major, so that for each c the block reads one
// contiguous column (lanes along r), as it reads the rows of hbi hii^-1:
// the element's 8 (NI + NE) NI bytes stream once from HBM, coalesced and
// evict-first, straight into the FMA chains; nothing is staged in shared
// memory but the two right-hand vectors, so many blocks share an SM and
// keep enough loads in flight.
template <int NP>
__global__ void __launch_bounds__(back_threads<NP>()) k_backsub(MeshView M, const Job *__restrict__ jobs) {
  constexpr int NN = NP * NP, NE = 4 * (NP - 1), NI = NN - NE, NT = back_threads<NP>();
  const Job J = jobs[blockIdx.y];
  const int e = blockIdx.x, tid = threadIdx.x;
  const int P = J.P;
  __shared__ double ub[2][NE], fi[2][NI];
  const size_t eo = (size_t)e * NN;
  const int *bt = M.btog + (size_t)e * NE;
  for (int b = tid; b < NE; b += NT) {
    const int g = bt[b];
    for (int p = 0; p < P; p++) ub[p][b] = (g < J.nsolve) ? J.rhs[(size_t)p * J.rhs_stride + g] : 0.0;
  }
  for (int i = tid; i < NI; i += NT)
    for (int p = 0; p < P; p++) fi[p][i] = J.f[(size_t)p * J.fstride + eo + NE + i];
  __syncthreads();
  // boundary values: the solved ones, then setEssential on masked nodes
  const bool masked = M.emask[e] != 0;
  for (int b = tid; b < NE; b += NT) {
    const int n = M.emap[b];
    const bool ess = masked && M.bmask[(size_t)e * NE + b];
    for (int p = 0; p < P; p++)
      J.u[(size_t)p * J.ustride + eo + n] = ess ? J.gess[(size_t)p * M.nglobal + bt[b]] : ub[p][b];
  }
  if (tid < NI) {
    const int r = tid;
    const double *hc = J.hii + (size_t)e * NI * NI + r;
    const double *hb = J.hbi + (size_t)e * NE * NI + r;
    double s0 = 0.0, s1 = 0.0, t0 = 0.0, t1 = 0.0;
    if (P > 1) {
#pragma unroll 9
      for (int c = 0; c < NI; c++) {
        const double v = __ldcs(hc + c * NI);
        s0 += v * fi[0][c];
        s1 += v * fi[1][c];
      }
#pragma unroll 8
      for (int b = 0; b < NE; b++) {
        const double v = __ldcs(hb + b * NI);
        t0 += v * ub[0][b];
        t1 += v * ub[1][b];
      }
    } else {
#pragma unroll 9
      for (int c = 0; c < NI; c++) s0 += __ldcs(hc + c * NI) * fi[0][c];
#pragma unroll 8
      for (int b = 0; b < NE; b++) t0 += __ldcs(hb + b * NI) * ub[0][b];
    }
    const int n = M.emap[NE + r];
    J.u[eo + n] = s0 - t0;
    if (P > 1) J.u[(size_t)J.ustride + eo + n] = s1 - t1;
  }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------

template <int NP>
static void launch_elem(const MeshView &M, const Job *djobs, int njobs, bool rhs, cudaStream_t st) {
  dim3 grid(M.nel, njobs);
  if (rhs)
    k_rhs_elem<NP><<<grid, ELEM_WARPS * 32, 0, st>>>(M, djobs);
  else
    k_backsub<NP><<<grid, back_threads<NP>(), 0, st>>>(M, djobs);
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
  if (M.np < 3 || M.np > 12) return SX_ERR_UNSUPPORTED;
  return prepare_band_kernels();
}

int direct_rhs_jobs(const MeshView &M, const Job *djobs, const std::vector<Job> &hjobs, cudaStream_t st,
                    int *launches) {
  const int nj = (int)hjobs.size();
  int maxpad = 0;
  bool any_bc = false;
  for (const Job &j : hjobs) {
    // the element kernels take both planes of a mode in one pass, no more
    if (j.P < 1 || j.P > 2) {
      set_error("direct solve: a job of %d planes (the element kernels take 1 or 2)", j.P);
      return SX_ERR_UNSUPPORTED;
    }
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
                      cudaStream_t st, const BandSched &sc, int *launches) {
  int nl = 0;
  SX_TRY(direct_rhs_jobs(M, djobs, hjobs, st, &nl));
  SX_TRY(band_sweep_jobs(djobs, hjobs, sc, st));
  SX_TRY(direct_backsub_jobs(M, djobs, (int)hjobs.size(), st, &nl));
  if (launches) *launches = nl + 1;
  return SX_OK;
}

}  // namespace sx
