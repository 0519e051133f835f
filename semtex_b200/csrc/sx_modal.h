// sx_modal.h -- the modal system object behind sx_modal (ModalMatrixSys) and
// its solve workspace; shared by the C ABI (sx_api.cu) and the serving loop
// (sx_serve.cu).
#pragma once

#include <functional>
#include <map>

#include "sx_internal.h"
#include "sx_kernels.cuh"
#include "sx_mixed.cuh"
#include "sx_pcg.cuh"
#include "sx_solve.cuh"

struct sx_modal_s {
  sx_mesh_s *mesh = nullptr;
  int base_mode = 0, num_modes = 0, method = SX_DIRECT;
  std::vector<std::shared_ptr<sx::System>> sys;   // per local mode
  std::vector<std::shared_ptr<sx::System>> uniq;  // distinct systems
  // solve workspace, sized for all planes at once
  sx::DBuf<double> rhs, Fb, gess;
  sx::PcgWork pcg;
  sx::DBuf<sx::Job> djobs;
  size_t npad_max = 0;
  // host-pointer entries: device staging
  sx::DBuf<double> hu, hf, hbc;
  // batched form: captured graph and the arguments it was captured for
  cudaStream_t own = nullptr;
  bool own_stream_external = false;
  cudaGraphExec_t gexec = nullptr;
  const void *gkey[3] = {nullptr, nullptr, nullptr};
  int gnz = 0, gstride = 0, gprec = -1;
  sx::DBuf<sx::Job> bjobs;
  std::vector<sx::Job> gjobs;        // host copy of the captured jobs
  int gC = 1, glaunches = 0;         // their band-sweep cluster size, kernel count
  sx::DBuf<int> dstatus;             // device status bits of the last solves
  // mixed-precision batched form
  sx::MixedWork mixed;
  const void *mkey[3] = {nullptr, nullptr, nullptr};
  int mnz = 0, mstride = 0;
  int n_inner = 12;                  // FP32 PCG iterations per refinement round
  bool use_graphs = true;
  std::map<int, int> cluster_for;    // jobs per launch -> band-sweep cluster size
  int forced_cluster = 0;
  int cluster(int nj);
  // Point this object at another mesh and set of systems, keeping the
  // workspace buffers (the serving loop reuses one object per slot).
  void rebind(sx_mesh_s *m, int base, int nmodes, int meth, std::vector<std::shared_ptr<sx::System>> s);
  ~sx_modal_s();
};

namespace sx {

// Supplies the system for (lambda2, betak2, kind) of a mode: builds it, or
// returns a cached one.  Returns a status.
using SystemProvider =
    std::function<int(double lambda2, double betak2, int kind, std::shared_ptr<System> &out)>;

// Fill M.sys / M.uniq for its modes (MIXED -> DIRECT for mode 0, JACPCG
// otherwise), factor the new DIRECT systems on stream st.
int modal_populate(sx_modal_s &M, const double *lam, const double *bk2, const SystemProvider *prov,
                   cudaStream_t st);

int solve_batched_on(sx_modal_s *s, double *d_u, double *d_f, const double *d_bc, int nz, int plane_stride,
                     int precision, double tol_rel, int max_refine, cudaStream_t st, sx_solve_stats *stats);

// Device -> host copy of the solved planes of a field (plane_stride doubles
// a plane).  The Nyquist plane (plane 1 when the base mode is 0 and nz > 1)
// is not solved and not copied: the caller's host plane stays as it was, as
// Field::solve leaves it (src/field.cpp:566).
int copy_solved_planes(double *h_u, const double *d_u, int nz, int plane_stride, int base_mode,
                       cudaStream_t st);

}  // namespace sx
