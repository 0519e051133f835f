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

namespace sx {

// A batched FP64 direct solve of a set of plane groups: the job table, and
// the kernel sequence captured once as a CUDA graph and replayed while the
// arguments it was captured for stay the same.
struct DirectBatch {
  cudaGraphExec_t exec = nullptr;
  const void *key[6] = {};  // u, f, bc, and the workspace buffers rhs, Fb, gess
  int nz = 0, stride = 0;
  std::vector<int> modes;  // local mode of each group, in job order
  DBuf<Job> djobs;
  std::vector<Job> jobs;   // host copy of the captured jobs
  BandSched sc;                   // band-sweep schedule
  int launches = 0;               // kernels per solve
  void reset() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    jobs.clear();
    modes.clear();
  }
  ~DirectBatch() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

}  // namespace sx

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
  // batched forms
  cudaStream_t own = nullptr;
  bool own_stream_external = false;
  sx::DirectBatch fp64;              // SX_FP64: every mode
  sx::DirectBatch hyb;               // SX_MIXED_FP32: the modes routed to the band solve
  cudaStream_t aux = nullptr;        // runs `hyb` beside the FP32 iterations
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  sx::DBuf<int> dstatus;             // device status bits of the last solves
  // mixed-precision batched form
  sx::MixedWork mixed;
  const void *mkey[3] = {nullptr, nullptr, nullptr};
  int mnz = 0, mstride = 0;
  std::vector<int> mmodes;           // local modes the FP32 iterations solve
  int n_inner = 12;                  // FP32 PCG iterations per refinement round, at least
  int mixed_route = 0;               // 0 auto, 1 FP32 CG only, 2 band solve where factored
  bool use_graphs = true;
  cudaMemPool_t pool = nullptr;      // when set, workspaces are allocated from it
  std::map<int, sx::BandSched> sched_for;  // systems per launch -> band-sweep schedule (default or tuned)
  int forced_cluster = 0, forced_stages = 0, forced_lead = -1;
  int host_chunk = 0;                // modes per host-pipeline chunk (0: auto)
  // Band-sweep schedule for nj systems per launch: the knobs where set, else
  // the autotuner's choice for nj, else the largest cluster whose CTAs are
  // all resident (and the default leader share).
  sx::BandSched sched(int nj);
  // host-buffer entry, pipelined: per-chunk views of this system (16 modes
  // each, sharing its systems) and the copy streams and events
  struct HostPipe {
    std::vector<std::unique_ptr<sx_modal_s>> views;
    cudaStream_t h2d = nullptr, d2h = nullptr;
    std::vector<cudaStream_t> cs;  // one per chunk: the chunks' solves run side by side
    std::vector<cudaEvent_t> in, done;
    ~HostPipe();
  };
  std::unique_ptr<HostPipe> pipe;
  // Point this object at another mesh and set of systems, keeping the
  // workspace buffers (the serving loop reuses one object per slot).
  void rebind(sx_mesh_s *m, int base, int nmodes, int meth, std::vector<std::shared_ptr<sx::System>> s);
  ~sx_modal_s();
};

// A multi-mesh batch (sx_batch_solve): the mixed-precision tables and
// graphs, and the direct solve whose band sweeps cover every member.
struct sx_batch_s {
  sx::MxBatch mixed;
  std::vector<long long> mkey;  // members and buffers the mixed tables were built for
  sx::DBuf<sx::Job> djobs;      // every member's direct jobs, member by member
  std::vector<sx::Job> jobs;
  std::vector<long long> dkey;  // members and buffers the direct graph was captured for
  cudaGraphExec_t dexec = nullptr;
  int dlaunches = 0;
  sx::BandSched sc;
  bool use_graphs = true;       // capture and replay (the serving loop, whose member set
                                // changes from batch to batch, enqueues directly)
  cudaStream_t own = nullptr, aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  ~sx_batch_s();
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

// SX_ERR_ARG (with a message naming `who`) unless the current device is the
// one the mesh -- and so every system built on it -- lives on.
int check_mesh_device(const sx_mesh_s &M, const char *who);

// Device -> host copy of the solved planes of a field (plane_stride doubles
// a plane).  The Nyquist plane (plane 1 when the base mode is 0 and nz > 1)
// is not solved and not copied: the caller's host plane stays as it was, as
// Field::solve leaves it (src/field.cpp:566).
int copy_solved_planes(double *h_u, const double *d_u, int nz, int plane_stride, int base_mode,
                       cudaStream_t st);

}  // namespace sx
