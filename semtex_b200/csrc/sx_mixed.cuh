// sx_mixed.cuh -- mixed-precision batched solve: FP32 Jacobi-PCG inner
// iterations wrapped in FP64 iterative refinement, all planes at once.
#pragma once

#include "sx_internal.h"

namespace sx {

// One plane of the batched mixed solve.
struct MxPlane {
  double *u;          // element plane (out)
  double *f;          // element plane (in, overwritten)
  const double *bc;   // nbound*np or nullptr
  double *gess;       // nglobal essential values
  const double *pc;   // npts FP64 inverse Jacobi diagonal
  const float *pcf;   // npts FP32 copy
  double hCon;
  int nsolve;
};

// Per-plane scalars (device): rho[2], pq[2], r2, b2, ...
struct MxScal {
  double rho[2];
  double pq[2];
  double r2, b2;
  double pad[2];
};

// Workspace + captured graphs for one batched plane set.
struct MixedWork {
  int planes = 0, npts = 0, n_inner = 0;
  DBuf<MxPlane> dplanes;
  DBuf<double> b64, x64, Ye64;
  DBuf<float> r32, d32, pA, pB, q32, Yb32;
  DBuf<MxScal> scal;
  DBuf<double> partA;   // per-plane block partials of the fused reductions
  DBuf<unsigned> cntA;  // per-plane "blocks finished" counters
  int maxblk = 0;
  cudaGraphExec_t g_init = nullptr, g_round = nullptr;
  int launches_init = 0, launches_round = 0;
  std::vector<MxScal> hscal;
  ~MixedWork() {
    if (g_init) cudaGraphExecDestroy(g_init);
    if (g_round) cudaGraphExecDestroy(g_round);
  }
};

// Run the batched mixed-precision solve.  Captures its graphs on first use
// (or when `rebuild`).  Stops when every plane's FP64 relative residual
// ||b - A x|| / ||b|| <= tol_rel or after max_refine rounds.
int mixed_solve(const MeshView &M, MixedWork &W, const std::vector<MxPlane> &planes, bool rebuild,
                double tol_rel, int max_refine, int n_inner, cudaStream_t st, sx_solve_stats *stats);

}  // namespace sx
