// sx_solve.cuh -- job descriptors and the element operator shared by the
// direct and iterative solve kernels.
#pragma once

#include "sx_internal.h"

namespace sx {

// A set of P planes sharing one system (P = 1 or 2: a Fourier mode's one
// or two planes).  Plane p of u / f / bc is at u + p*ustride etc.
struct Job {
  double *u;
  double *f;
  const double *bc;
  long long ustride, fstride, bcstride;
  int P;
  double hCon;          // lambda2 + betak2
  int nsolve;           // system nsolve (reduced by one when singular)
  // DIRECT
  const double *hbi, *hii;
  const double *tiles, *dinv;
  int nblk, J, npad;
  const int *jf, *jb;   // factor envelope by block column / row (null: whole band)
  double *rhs;          // P * rhs_stride
  long long rhs_stride;
  double *Fb;           // P * nel * next
  double *gess;         // P * nglobal
  // JACPCG
  const double *pc;
  int *status;          // device status bits (1 << SX_ERR_*)
};

// out = A_e u for one element (Element::HelmholtzOp + HelmholtzKern,
// src/element.cpp:1564-1650, Cartesian): R = u DT, S = D u, pointwise
// geometric factors, out = Q4 u hCon + DT S + R D.  All arrays np*np
// row-major in shared memory; ends with __syncthreads().
template <int NP, typename T>
__device__ __forceinline__ void helm_op(const T *D, const T *Q1, const T *Q2, const T *Q3, const T *Q4,
                                        bool q3, T hCon, const T *u, T *R, T *S, T *out, int nthreads) {
  constexpr int NN = NP * NP;
  for (int idx = threadIdx.x; idx < NN; idx += nthreads) {
    const int i = idx / NP, j = idx - i * NP;
    T r = 0, s = 0;
#pragma unroll
    for (int k = 0; k < NP; k++) {
      r += u[i * NP + k] * D[j * NP + k];
      s += D[i * NP + k] * u[k * NP + j];
    }
    if (q3) {
      R[idx] = Q1[idx] * r + Q3[idx] * s;
      S[idx] = Q2[idx] * s + Q3[idx] * r;
    } else {
      R[idx] = Q1[idx] * r;
      S[idx] = Q2[idx] * s;
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < NN; idx += nthreads) {
    const int i = idx / NP, j = idx - i * NP;
    T t = Q4[idx] * u[idx] * hCon;
    T a = 0, b = 0;
#pragma unroll
    for (int k = 0; k < NP; k++) {
      a += D[k * NP + i] * S[k * NP + j];
      b += R[i * NP + k] * D[k * NP + j];
    }
    out[idx] = t + a + b;
  }
  __syncthreads();
}

// Direct solve of all jobs; the band sweeps run one cluster of C CTAs per job.
// Returns the number of kernels launched through *launches when non-null.
// Ring depth (tiles in flight per CTA) of the band sweeps: at most 4; 2
// lets two CTAs share an SM, so that larger clusters stay resident.
constexpr int BAND_STAGES_MAX = 4;
// Schedule of one band-sweep launch: C CTAs per system's cluster, S tiles in
// flight per CTA, and the leader's share of the tiles j >= 2: Q = 0 none,
// Q = K >= 2 the last of every K of them (worked on a step ahead).
struct BandSched {
  int C = 1, S = BAND_STAGES_MAX, Q = 0;
  bool operator==(const BandSched &o) const { return C == o.C && S == o.S && Q == o.Q; }
};
int direct_solve_jobs(const MeshView &M, const Job *djobs, const std::vector<Job> &hjobs,
                      cudaStream_t st, const BandSched &sc, int *launches = nullptr);
// The phases of direct_solve_jobs, for batches whose band sweeps run in one
// launch across meshes: essential values, condensed RHS (element kernels
// and direct-stiffness sum); then, after the sweeps, the interior
// back-substitution.  Each adds its launches to *launches when non-null.
int direct_rhs_jobs(const MeshView &M, const Job *djobs, const std::vector<Job> &hjobs, cudaStream_t st,
                    int *launches);
int direct_backsub_jobs(const MeshView &M, const Job *djobs, int nj, cudaStream_t st, int *launches);
int band_sweep_jobs(const Job *djobs, const std::vector<Job> &hjobs, const BandSched &sc, cudaStream_t st);
int prepare_band_kernels();
// Bounded device-side waits on the current device (sx_set_wait_limit): the
// band sweeps' and the FP32 iterations' limits in clock cycles (<= 0: one
// probe).
constexpr long long SWEEP_WAIT_DEFAULT = 4000000000LL, CG_WAIT_DEFAULT = 2000000000LL;
int set_sweep_wait_limit(long long cycles);
int set_cg_wait_limit(long long cycles);
int pick_cluster(int nj, int cmax, int pmax, int Wmax, int *stages_out = nullptr, int stages_forced = 0);
// Default leader share Q (0 or a cycle length K >= 2) of a cluster of C CTAs
// on a band of J off-diagonal tiles per block column.
int default_lead(int C, int J);
// Clusters of C band-sweep CTAs that can be resident at once (0: C does not
// fit an SM group, so a launch with it would fail).
int band_active_clusters(int C, int pmax, int Wmax, int stages = BAND_STAGES_MAX);
size_t sweep_smem(int pmax, int C, int S, int Wmax);
// Set kernel attributes (max dynamic smem) ahead of any stream capture.
int prepare_direct_kernels(const MeshView &M);

}  // namespace sx
