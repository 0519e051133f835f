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
  const int *active;    // [PP] 1 for planes this form solves (not the Nyquist
                        // plane, padding, or planes routed to the direct path)
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

// Per-plane scalars, each an array of PP doubles: residual and RHS norms
// (read by the host between rounds), then the inner iteration's gamma,
// alpha, beta in two slots (iteration parity), and gamma at the start of the
// round.
constexpr int MX_NSCAL = 9;
struct MxScalPtrs {
  double *r2, *b2, *gam[2], *alpha[2], *beta[2], *gam0;
};

// Vectors of the FP32 inner iteration in element layout ("E-vectors"): every
// element keeps its own copy of its nodes' values, chunk-major,
// V[((e * nch + y) * np^2 + t) * 32 + l] for element e, plane chunk y,
// tensor node t and lane (plane) l, so one block's data is one contiguous
// np^2 * 128-byte span that a single TMA bulk copy moves.  The copies of a
// shared node are updated by every element that holds it, with the same
// arithmetic on the same inputs, so they stay equal; r, s, p, d are read and
// written only by their element's block and stay in place.  A u is gathered
// across elements, so it alternates between two buffers by parity.
struct CgVecs {
  float *rE, *sE, *pE, *dE;
  float *WE[2];       // A u at every element node (unassembled)
  const float *pcE;   // inverse Jacobi diagonal, [e][y][t][16] by mode pair
  const float *r0;    // residual of the last refinement step, [npts][PP]
  double *x64;
  double *gam[2], *alpha[2], *beta[2];
  double *gam0;       // gamma at the start of the round
  int *status;        // device status bits (1 << SX_ERR_*)
};

struct MixedWork {
  int PP = 0, npts = 0, n_inner = 0, M = 0, G = 0;
  DBuf<double> hcon, b64, x64, Ye64, scal, part, gess;
  DBuf<int> nsolve, active;
  DBuf<unsigned> cnt;
  DBuf<float> pcf, r0, rE, sE, pE, dE, WE0, WE1, pcE;
  int *status = nullptr;  // the owner's device status word
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

// Run the batched mixed-precision solve of the planes of `groups` (nz
// planes in the caller's arrays; the others -- the Nyquist plane, planes
// solved by another path -- are neither read nor written).  Stops when every
// plane's FP64 relative residual ||b - A x|| / ||b|| <= tol_rel or after
// max_refine rounds.
int mixed_solve(const MeshView &M, MixedWork &W, const std::vector<MxGroup> &groups, int nz, int num_modes,
                double *d_u, double *d_f, const double *d_bc, long long stride, bool rebuild, double tol_rel,
                int max_refine, int n_inner, bool graphs, cudaStream_t st, sx_solve_stats *stats);

// Enqueue `reps` inner-iteration launches (k_cg, iteration 1) on the
// workspace of the last mixed solve, for timing the kernel on its own.  The
// workspace's iterates are left meaningless; the next solve starts afresh.
int mixed_profile_iterations(const MeshView &M, MixedWork &W, int reps, cudaStream_t st);

}  // namespace sx
