// sx_pcg.cuh -- Jacobi-preconditioned CG on the GPU (declarations).
#pragma once

#include "sx_internal.h"
#include "sx_solve.cuh"

namespace sx {

// Workspace for one plane's PCG (vectors of npts = nglobal + nel*nint).
struct PcgWork {
  int npts = 0;
  DBuf<double> r, p, q, x, Ye, part, scal;
  int reserve(const MeshView &M);
};

// Solve every plane of `job` with the reference's JACPCG iteration
// (src/field.cpp:627-720).  Returns SX_OK or SX_WARN_STEP_LIMIT.
int pcg_solve_job(const MeshView &M, const System &S, PcgWork &W, const Job &job, double tol_rel,
                  int step_max, cudaStream_t st, int *iters_max, double *rel_res, int *launches);

// y = A x on global vectors (Field::HelmholtzOperator, src/field.cpp:771-856).
int global_op(const MeshView &M, double hCon, const double *x, double *y, double *Ye, cudaStream_t st);

}  // namespace sx
