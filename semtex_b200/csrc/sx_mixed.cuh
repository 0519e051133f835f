// sx_mixed.cuh -- mixed-precision batched solve: FP32 Jacobi-PCG inner
// iterations wrapped in FP64 iterative refinement, all planes at once, on
// plane-interleaved vectors.
#pragma once

#include "sx_internal.h"

namespace sx {

constexpr int MX_CH = 32;  // planes per block chunk (one warp lane per plane)

// Per-solve constants (device side).
struct MxParams {
  int PP;               // padded plane count (multiple of MX_CH)
  int nz;               // real planes in the caller's arrays
  int nyq;              // Nyquist plane (not solved) or -1
  int M;                // columns of the interleaved preconditioner (local modes)
  const double *hcon;   // [PP] lambda2 + betak2 of the plane's mode
  const int *nsolve;    // [PP]
  const float *pcf;     // [npts * M] inverse Jacobi diagonal, mode-interleaved
  const double *f;      // forcing planes (plane-major, caller layout)
  double *u;            // solution planes
  long long stride;     // plane stride of f and u
  const double *bc;     // bc lines per plane or nullptr
  long long bcstride;
  double *gess;         // [PP * nglobal] essential values, plane-major
};

// Per-plane scalars, each an array of PP doubles.
struct MxScalPtrs {
  double *rho0, *rho1, *pq0, *pq1, *r2, *b2;
};

struct MixedWork {
  int PP = 0, npts = 0, n_inner = 0, M = 0, G = 0;
  DBuf<double> hcon, b64, x64, Ye64, scal, part, gess;
  DBuf<int> nsolve;
  DBuf<unsigned> cnt;
  DBuf<float> pcf, r32, d32, pA, pB, q32, Yb32;
  cudaGraphExec_t g_init = nullptr, g_round = nullptr;
  int launches_init = 0, launches_round = 0;
  std::vector<double> hscal;
  MxParams prm{};
  ~MixedWork() {
    if (g_init) cudaGraphExecDestroy(g_init);
    if (g_round) cudaGraphExecDestroy(g_round);
  }
};

// One plane group of the batched solve: planes [plane0, plane0 + P) use
// the system of local mode `mode`.
struct MxGroup {
  int mode, plane0, P;
  const System *sys;
};

// Run the batched mixed-precision solve of planes 0..nz-1 (plane 1 is the
// Nyquist datum when nyq == 1).  Stops when every plane's FP64 relative
// residual ||b - A x|| / ||b|| <= tol_rel or after max_refine rounds.
int mixed_solve(const MeshView &M, MixedWork &W, const std::vector<MxGroup> &groups, int nz, int nyq,
                int num_modes, double *d_u, double *d_f, const double *d_bc, long long stride, bool rebuild,
                double tol_rel, int max_refine, int n_inner, bool graphs, cudaStream_t st,
                sx_solve_stats *stats);

}  // namespace sx
