// sx_mixed.cuh -- mixed-precision batched solve: FP32 Jacobi-PCG inner
// iterations wrapped in FP64 iterative refinement, all planes at once, on
// plane-interleaved vectors.
#pragma once

#include <vector>

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
  float *r0;          // residual of the last refinement step, [npts][PP]
  double *x64;
  double *gam[2], *alpha[2], *beta[2];
  double *gam0;       // gamma at the start of the round
  int *status;        // device status bits (1 << SX_ERR_*)
  // per plane chunk: 1 when every plane of the chunk has stopped for the
  // rest of the round (alpha = beta = 0), so the chunk's blocks skip the
  // following iterations; written by each launch's reduction for the next
  int *skip;
};

// Everything the kernels of one solve read and write: the mesh, the
// per-plane constants, the CG vectors and scalars, and the reduction
// scratch.  A single-mesh solve passes it as a kernel parameter; a
// multi-mesh batch keeps one per member in device memory.
struct MxMember {
  MeshView M;
  MxParams P;
  CgVecs V;
  double *Ye, *b64;  // FP64 element results, FP64 RHS [npts][PP]
  double *r2, *b2;   // per-plane ||r||^2 and ||b||^2, read by the host
  double *part;      // reduction partials
  unsigned *cnt;     // reduction counters
  int nch;           // plane chunks of 32 (P.PP / 32)
  int G;             // blocks per chunk of the node kernels
};

struct MixedWork {
  int PP = 0, npts = 0, n_inner = 0, M = 0, G = 0;
  DBuf<double> hcon, b64, x64, Ye64, scal, part, gess;
  DBuf<int> nsolve, active, skip;
  DBuf<unsigned> cnt;
  DBuf<float> pcf, r0, rE, sE, pE, dE, WE0, WE1, pcE;
  int *status = nullptr;  // the owner's device status word
  cudaGraphExec_t g_init = nullptr, g_round = nullptr;
  int launches_init = 0, launches_round = 0;
  // setup() counts its runs here; a captured graph (this workspace's own,
  // or a batch's) is valid while the count it was captured at still holds
  unsigned epoch = 0, graph_epoch = 0;
  bool check_stop = false;  // the captured round reads the chunks' stop flags
  cudaMemPool_t pool = nullptr;  // when set, setup() allocates from it
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
// check_stop: the FP32 iterations read each chunk's stop flag, so that
// chunks whose planes have all stopped skip the rest of the round (worth
// its latency when some planes need far fewer iterations than the round).
int mixed_solve(const MeshView &M, MixedWork &W, const std::vector<MxGroup> &groups, int nz, int num_modes,
                double *d_u, double *d_f, const double *d_bc, long long stride, bool rebuild, double tol_rel,
                int max_refine, int n_inner, bool check_stop, bool graphs, cudaStream_t st,
                sx_solve_stats *stats);

// One member of a multi-mesh mixed-precision solve: a mesh, its workspace
// and plane groups, and the caller's arrays.  `stats` is filled on return.
struct MxItem {
  MeshView M;
  MixedWork *W = nullptr;
  std::vector<MxGroup> groups;
  int nz = 0, num_modes = 0;
  double *u = nullptr, *f = nullptr;
  const double *bc = nullptr;
  long long stride = 0;
  sx_solve_stats stats{};
};

// Device tables, streams and graphs of a multi-mesh mixed-precision solve.
// Members are ordered by element order; the members of one order form a
// class, and every kernel runs once per class over all its members' tiles
// (element tiles: nel * nch per member; node tiles: G * nch; plane tiles:
// PP), the classes on their own streams side by side.
struct MxBatch {
  struct Class {
    int np = 0, m0 = 0, count = 0;  // order, first member, members
    int te = 0, tn = 0, tp = 0;     // element, node and plane tiles
    size_t t0 = 0;                  // offset of the 3 (count + 1) tile prefixes
  };
  DBuf<MxMember> mem;
  DBuf<int> tiles;
  DBuf<double> norms;             // r2 then b2 of each member, PP each
  std::vector<Class> cls;
  std::vector<int> order;         // item index of each member
  std::vector<size_t> noff;       // each member's offset in norms
  std::vector<unsigned> epochs;   // each member workspace's epoch after setup
  std::vector<double> hnorms;
  std::vector<cudaStream_t> streams;  // one per class
  std::vector<cudaEvent_t> events;    // fork + one join per class
  cudaGraphExec_t g_init = nullptr, g_round = nullptr;
  int launches_init = 0, launches_round = 0, n_inner = 0;
  bool check_stop = false;
  void reset();
  ~MxBatch();
};

// Solve every item's plane groups in one batch: each refinement round is
// one graph whose kernels cover the tiles of all members (one launch per
// kernel and element order).  Rounds continue until every plane of every
// member meets tol_rel, or max_refine.  Returns SX_WARN_STEP_LIMIT when a
// member did not converge.
int mixed_solve_multi(std::vector<MxItem> &items, MxBatch &B, bool rebuild, double tol_rel, int max_refine,
                      int n_inner, bool check_stop, bool graphs, cudaStream_t st);

// Enqueue `reps` inner-iteration launches (k_cg, iteration 1) on the
// workspace of the last mixed solve, for timing the kernel on its own.  The
// workspace's iterates are left meaningless; the next solve starts afresh.
int mixed_profile_iterations(const MeshView &M, MixedWork &W, int reps, cudaStream_t st);

}  // namespace sx
