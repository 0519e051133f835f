// sx_api.cu -- C ABI: ModalMatrixSys and Field::solve replacements.
#include <cmath>
#include <cstring>

#include "sx_modal.h"

namespace sx {
const char *last_error();
}

using namespace sx;

// ---------------------------------------------------------------------------
// sx_modal_s
// ---------------------------------------------------------------------------

BandSched sx_modal_s::sched(int nj) {
  int J = 1;
  for (auto &s : uniq) J = std::max(J, s->J);
  BandSched sc;
  if (forced_cluster > 0) {
    sc.C = forced_cluster;
    sc.S = forced_stages > 0 ? forced_stages : BAND_STAGES_MAX;
    sc.Q = default_lead(sc.C, J);
  } else {
    auto it = sched_for.find(nj);
    if (it != sched_for.end()) {
      sc = it->second;
    } else {
      // ranks 1..C-1 share the J-1 tiles j >= 2, so C <= J
      sc.C = pick_cluster(nj, std::min(16, std::max(1, J)), 2, J + 2, &sc.S, forced_stages);
      sc.Q = default_lead(sc.C, J);
      sched_for[nj] = sc;
    }
  }
  if (forced_lead >= 0) sc.Q = forced_lead;
  return sc;
}

void sx_modal_s::rebind(sx_mesh_s *m, int base, int nmodes, int meth, std::vector<std::shared_ptr<System>> s) {
  mesh = m;
  base_mode = base;
  num_modes = nmodes;
  method = meth;
  sys = std::move(s);
  uniq.clear();
  for (auto &x : sys)
    if (std::find(uniq.begin(), uniq.end(), x) == uniq.end()) uniq.push_back(x);
  fp64.reset();
  hyb.reset();
  mkey[0] = mkey[1] = mkey[2] = nullptr;
  mmodes.clear();
  sched_for.clear();
}

sx_modal_s::~sx_modal_s() {
  fp64.reset();
  hyb.reset();
  if (ev_fork) cudaEventDestroy(ev_fork);
  if (ev_join) cudaEventDestroy(ev_join);
  if (aux) cudaStreamDestroy(aux);
  if (own && !own_stream_external) cudaStreamDestroy(own);
}

extern "C" const char *sx_version(void) { return "semtex_b200 0.2 (sm_100a)"; }

extern "C" const char *sx_status_string(int s) {
  switch (s) {
    case SX_OK: return "ok";
    case SX_ERR_ARG: return "invalid argument";
    case SX_ERR_CUDA: return "CUDA error";
    case SX_ERR_NOMEM: return "out of memory";
    case SX_ERR_JACOBIAN: return "nonpositive element Jacobian";
    case SX_ERR_SINGULAR_HII: return "singular interior matrix hii";
    case SX_ERR_NOT_SPD: return "failed to factor Helmholtz matrix";
    case SX_ERR_BAND: return "numbering exceeds declared band";
    case SX_WARN_STEP_LIMIT: return "PCG step limit exceeded";
    case SX_ERR_UNSUPPORTED: return "unsupported configuration";
    case SX_ERR_TIMEOUT: return "device wait timed out";
    case SX_ERR_CAPACITY: return "request exceeds memory budget";
    case SX_ERR_NOT_FOUND: return "unknown request";
    default: return "unknown status";
  }
}

extern "C" const char *sx_last_error(void) { return last_error(); }

extern "C" int sx_set_device(int device) {
  SX_CUDA(cudaSetDevice(device));
  return SX_OK;
}

extern "C" int sx_set_wait_limit(double ms) {
  long long sweep = SWEEP_WAIT_DEFAULT, cg = CG_WAIT_DEFAULT;
  if (ms >= 0.0) {
    int dev = 0, khz = 0;
    SX_CUDA(cudaGetDevice(&dev));
    SX_CUDA(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev));
    sweep = cg = (long long)(ms * (double)khz);  // clock64 counts SM cycles
  }
  SX_TRY(set_sweep_wait_limit(sweep));
  SX_TRY(set_cg_wait_limit(cg));
  return SX_OK;
}

static bool same_constants(const System &S, double lambda2, double betak2, int method) {
  // MatrixSys::match, src/matrix.cpp:326-347 (same mesh numbering implied).
  return std::fabs(S.lambda2 - lambda2) < EPSDP && std::fabs(S.betak2 - betak2) < EPSDP &&
         S.method == method;
}

namespace sx {

int modal_populate(sx_modal_s &M, const double *lam, const double *bk2, const SystemProvider *prov,
                   cudaStream_t st) {
  std::vector<System *> to_factor;
  M.sys.clear();
  M.uniq.clear();
  for (int l = 0; l < M.num_modes; l++) {
    const int mode = M.base_mode + l;
    int kind = M.method;
    if (M.method == SX_MIXED) kind = (mode == 0) ? SX_DIRECT : SX_JACPCG;  // src/matrix.cpp:93-96
    if (M.method == SX_AUTO) {
      // a modal system is built to be solved many times (a DNS run solves
      // it every timestep): the factorisation is charged over 100 solves;
      // 1e-12 in at most 20 rounds is the batched form's default target
      const sx_mesh_s &Mh = *M.mesh;
      kind = band_cheaper(Mh.np, Mh.nel, Mh.nglobal, Mh.nsolve, Mh.nband, Mh.kratio, lam[l] + bk2[l], M.n_inner,
                          1e-12, 20, 100.0)
                 ? SX_DIRECT
                 : SX_JACPCG;
    }
    std::shared_ptr<System> found;
    for (auto &s : M.uniq)
      if (same_constants(*s, lam[l], bk2[l], kind)) {
        found = s;
        break;
      }
    if (!found && prov) {
      SX_TRY((*prov)(lam[l], bk2[l], kind, found));
    } else if (!found) {
      found = std::make_shared<System>();
      found->mesh = M.mesh;
      found->lambda2 = lam[l];
      found->betak2 = bk2[l];
      found->method = kind;
      if (kind == SX_DIRECT) {
        SX_TRY(system_build_direct(*found, st));
        if (found->nsolve > 0) to_factor.push_back(found.get());
      } else {
        SX_TRY(system_build_jacobi(*found, st));
      }
    }
    if (std::find(M.uniq.begin(), M.uniq.end(), found) == M.uniq.end()) M.uniq.push_back(found);
    M.sys.push_back(found);
  }
  if (!M.dstatus.p) {
    SX_TRY(M.dstatus.alloc(1));
    SX_TRY(M.dstatus.zero(st));
  }
  SX_TRY(factor_batch(to_factor, st));
  for (System *S : to_factor) {
    int h = 0;
    SX_CUDA(cudaMemcpyAsync(&h, S->status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SX_CUDA(cudaStreamSynchronize(st));
    if (h & (1 << SX_ERR_NOT_SPD)) {
      set_error("failed to factor Helmholtz matrix (lambda2=%g, betak2=%g)", S->lambda2, S->betak2);
      return SX_ERR_NOT_SPD;
    }
  }
  return SX_OK;
}

}  // namespace sx

static int modal_build(sx_mesh m, int base_mode, int num_modes, const double *lam, const double *bk2,
                       int method, sx_modal *out) {
  if (!m || !out || num_modes <= 0 || base_mode < 0 || method < SX_DIRECT || method > SX_AUTO)
    return SX_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<sx_modal_s> M(new sx_modal_s());
  M->mesh = m;
  M->base_mode = base_mode;
  M->num_modes = num_modes;
  M->method = method;
  SX_TRY(modal_populate(*M, lam, bk2, nullptr, 0));
  *out = M.release();
  return SX_OK;
}

extern "C" int sx_modal_create(sx_mesh m, double lambda2, double beta, int base_mode, int num_modes,
                               int method, sx_modal *out) {
  if (num_modes <= 0) return SX_ERR_ARG;
  std::vector<double> lam(num_modes, lambda2), bk2(num_modes);
  for (int l = 0; l < num_modes; l++) {
    const double bk = beta * (base_mode + l);  // Field::modeConstant, Cartesian
    bk2[l] = bk * bk;
  }
  return modal_build(m, base_mode, num_modes, lam.data(), bk2.data(), method, out);
}

extern "C" int sx_modal_create_ex(sx_mesh m, int base_mode, int num_modes, const double *lambda2,
                                  const double *betak2, int method, sx_modal *out) {
  if (!lambda2 || !betak2) return SX_ERR_ARG;
  return modal_build(m, base_mode, num_modes, lambda2, betak2, method, out);
}

extern "C" int sx_modal_destroy(sx_modal s) {
  delete s;
  return SX_OK;
}

extern "C" int sx_modal_band(sx_modal s, int m, double *ab, int *nsolve, int *singular) {
  if (!s || m < 0 || m >= s->num_modes) return SX_ERR_ARG;
  const System &S = *s->sys[m];
  if (nsolve) *nsolve = S.nsolve;
  if (singular) *singular = S.singular ? 1 : 0;
  if (S.method != SX_DIRECT) return SX_ERR_ARG;
  if (ab) SX_TRY(system_band_export(S, ab));
  return SX_OK;
}

// Device-side status of the solves enqueued so far (bounded waits that ran
// out, ...).  Synchronises `st` (the whole device when st is null) and
// clears the word when `clear`.
static int take_status(sx_modal s, bool clear, cudaStream_t st = nullptr, bool device = true) {
  int h = 0;
  if (device)
    SX_CUDA(cudaDeviceSynchronize());
  else
    SX_CUDA(cudaStreamSynchronize(st));
  SX_CUDA(cudaMemcpyAsync(&h, s->dstatus.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  SX_CUDA(cudaStreamSynchronize(st));
  if (clear && h) SX_CUDA(cudaMemsetAsync(s->dstatus.p, 0, sizeof(int), st));
  if (h & (1 << SX_ERR_TIMEOUT)) {
    set_error("a bounded device-side wait ran out (band sweep)");
    return SX_ERR_TIMEOUT;
  }
  return SX_OK;
}

extern "C" int sx_modal_tune(sx_modal s, int knob, int value) {
  if (!s) return SX_ERR_ARG;
  switch (knob) {
    case SX_TUNE_INNER_ITERS:
      if (value > 1000) return SX_ERR_ARG;
      s->n_inner = value > 0 ? value : 12;
      return SX_OK;
    case SX_TUNE_BAND_CLUSTER:
      if (value > 16) return SX_ERR_ARG;
      s->forced_cluster = value > 0 ? value : 0;
      s->fp64.reset();  // the captured graphs bake in the cluster size
      s->hyb.reset();
      return SX_OK;
    case SX_TUNE_MIXED_ROUTE:
      if (value < 0 || value > 2) return SX_ERR_ARG;
      s->mixed_route = value;
      return SX_OK;
    case SX_TUNE_BAND_STAGES:
      if (value < 0 || value > BAND_STAGES_MAX) return SX_ERR_ARG;
      s->forced_stages = value > 0 ? value : 0;
      s->sched_for.clear();
      s->fp64.reset();
      s->hyb.reset();
      return SX_OK;
    case SX_TUNE_HOST_CHUNK:
      if (value > 1 << 20) return SX_ERR_ARG;
      s->host_chunk = value > 0 ? value : 0;
      return SX_OK;
    case SX_TUNE_BAND_LEAD:
      if (value > 64) return SX_ERR_ARG;
      s->forced_lead = value <= 0 ? -1 : (value == 1 ? 0 : value);
      s->fp64.reset();
      s->hyb.reset();
      return SX_OK;
    default:
      return SX_ERR_ARG;
  }
}

extern "C" int sx_modal_status(sx_modal s) {
  if (!s) return SX_ERR_ARG;
  return take_status(s, true);
}

extern "C" unsigned long long sx_modal_device_bytes(sx_modal s) {
  if (!s) return 0;
  size_t b = 0;
  for (auto &u : s->uniq) b += u->bytes();
  return b;
}

// Plane groups of a solve: local mode l owns planes 2l, 2l+1; plane 1 is the
// Nyquist datum when the base mode is 0 (src/field.cpp:564-573).
struct Group {
  int mode;    // local mode
  int plane0;  // first plane
  int P;       // planes
};

static int plane_groups(const sx_modal_s &M, int nz, std::vector<Group> &g) {
  g.clear();
  if (nz <= 0) return SX_ERR_ARG;
  if (nz == 1) {
    g.push_back({0, 0, 1});
    return SX_OK;
  }
  if (nz % 2) return SX_ERR_ARG;
  if (nz / 2 > M.num_modes) return SX_ERR_ARG;
  for (int l = 0; l < nz / 2; l++) {
    if (l == 0 && M.base_mode == 0)
      g.push_back({0, 0, 1});
    else
      g.push_back({l, 2 * l, 2});
  }
  return SX_OK;
}

// Workspace for `planes` planes; reallocates only what is too small (the
// serving loop reuses one workspace across meshes).
static int reserve_ws(sx_modal_s &M, int planes) {
  const sx_mesh_s &Mh = *M.mesh;
  size_t npad = 1;
  for (auto &s : M.uniq) npad = std::max(npad, (size_t)std::max(s->nblk, 1) * NB);
  M.npad_max = npad;
  cudaStream_t st = M.own;
  if (M.rhs.n < (size_t)planes * npad) SX_TRY(M.rhs.alloc_in((size_t)planes * npad, M.pool, st));
  if (M.Fb.n < (size_t)planes * Mh.nel * Mh.next)
    SX_TRY(M.Fb.alloc_in((size_t)planes * Mh.nel * Mh.next, M.pool, st));
  if (M.gess.n < (size_t)planes * Mh.nglobal) SX_TRY(M.gess.alloc_in((size_t)planes * Mh.nglobal, M.pool, st));
  return SX_OK;
}

static Job make_job(sx_modal_s &M, const Group &g, int slot, double *u, double *f, const double *bc,
                    long long stride, long long bcstride) {
  const sx_mesh_s &Mh = *M.mesh;
  const System &S = *M.sys[g.mode];
  Job j;
  std::memset(&j, 0, sizeof(j));
  j.u = u + (long long)g.plane0 * stride;
  j.f = f + (long long)g.plane0 * stride;
  j.bc = bc ? bc + (long long)g.plane0 * bcstride : nullptr;
  j.ustride = j.fstride = stride;
  j.bcstride = bcstride;
  j.P = g.P;
  j.hCon = S.betak2 + S.lambda2;
  j.nsolve = S.nsolve;
  j.hbi = S.hbi.p;
  j.hii = S.hii.p;
  j.tiles = S.tiles.p;
  j.dinv = S.dinv.p;
  j.nblk = S.nblk;
  j.J = S.J;
  j.jf = S.mesh->denv.p;
  j.jb = S.mesh->denv.p + S.mesh->env_nblk;
  j.npad = std::max(S.nblk, 1) * NB;
  j.rhs_stride = (long long)M.npad_max;
  j.rhs = M.rhs.p + (size_t)slot * M.npad_max;
  j.Fb = M.Fb.p + (size_t)slot * Mh.nel * Mh.next;
  j.gess = M.gess.p + (size_t)slot * Mh.nglobal;
  j.pc = S.pc.p;
  j.status = M.dstatus.p;
  return j;
}

extern "C" int sx_field_solve_device(sx_modal s, double *d_u, double *d_f, const double *d_bc, int nz,
                                     int plane_stride, double tol_rel, int step_max, void *stream,
                                     sx_solve_stats *stats) {
  if (!s || !d_u || !d_f || plane_stride < s->mesh->nel * s->mesh->npnp) return SX_ERR_ARG;
  SX_TRY(check_mesh_device(*s->mesh, "sx_field_solve_device"));
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<Group> groups;
  SX_TRY(plane_groups(*s, nz, groups));
  int planes = 0;
  for (auto &g : groups) planes += g.P;
  SX_TRY(reserve_ws(*s, planes));
  const long long bcstride = (long long)std::max(s->mesh->nbound, 1) * s->mesh->np;
  std::vector<Job> jobs;
  int slot = 0;
  for (auto &g : groups) {
    jobs.push_back(make_job(*s, g, slot, d_u, d_f, d_bc, plane_stride, bcstride));
    slot += g.P;
  }
  if (s->djobs.n < jobs.size()) SX_TRY(s->djobs.alloc(jobs.size()));
  SX_CUDA(cudaMemcpyAsync(s->djobs.p, jobs.data(), jobs.size() * sizeof(Job), cudaMemcpyHostToDevice, st));
  const MeshView M = s->mesh->view();
  SX_TRY(prepare_direct_kernels(M));
  sx_solve_stats loc{};
  int rc = SX_OK;
  // Mode by mode, as Field::solve's plane loop.
  for (size_t i = 0; i < groups.size(); i++) {
    const System &S = *s->sys[groups[i].mode];
    std::vector<Job> one(1, jobs[i]);
    if (S.method == SX_DIRECT) {
      int nl = 0;
      SX_TRY(direct_solve_jobs(M, s->djobs.p + i, one, st, s->sched(1), &nl));
      loc.kernel_launches += nl;
    } else {
      int iters = 0;
      double rr = 0.0;
      const int r = pcg_solve_job(M, S, s->pcg, jobs[i], tol_rel, step_max, st, &iters, &rr,
                                  &loc.kernel_launches);
      if (r != SX_OK && r != SX_WARN_STEP_LIMIT) return r;
      if (r == SX_WARN_STEP_LIMIT) rc = SX_WARN_STEP_LIMIT;
      loc.iterations_max = std::max(loc.iterations_max, iters);
      loc.iterations_total += iters * groups[i].P;
      loc.final_rel_residual = std::max(loc.final_rel_residual, rr);
    }
    loc.planes_solved += groups[i].P;
  }
  SX_CUDA(cudaGetLastError());
  if (stats) *stats = loc;
  return rc;
}

extern "C" int sx_field_solve(sx_modal s, double *u, double *f, const double *bc, int nz, int plane_stride,
                              double tol_rel, int step_max, sx_solve_stats *stats) {
  if (!s || !u || !f || nz <= 0) return SX_ERR_ARG;
  SX_TRY(check_mesh_device(*s->mesh, "sx_field_solve"));
  const size_t n = (size_t)nz * plane_stride;
  const size_t nbc = (size_t)nz * std::max(s->mesh->nbound, 1) * s->mesh->np;
  if (s->hu.n < n) SX_TRY(s->hu.alloc(n));
  if (s->hf.n < n) SX_TRY(s->hf.alloc(n));
  if (bc && s->hbc.n < nbc) SX_TRY(s->hbc.alloc(nbc));
  SX_CUDA(cudaMemcpy(s->hu.p, u, n * 8, cudaMemcpyHostToDevice));
  SX_CUDA(cudaMemcpy(s->hf.p, f, n * 8, cudaMemcpyHostToDevice));
  if (bc) SX_CUDA(cudaMemcpy(s->hbc.p, bc, nbc * 8, cudaMemcpyHostToDevice));
  const int rc = sx_field_solve_device(s, s->hu.p, s->hf.p, bc ? s->hbc.p : nullptr, nz, plane_stride,
                                       tol_rel, step_max, nullptr, stats);
  if (rc != SX_OK && rc != SX_WARN_STEP_LIMIT) return rc;
  SX_TRY(take_status(s, true));
  SX_CUDA(cudaMemcpy(u, s->hu.p, n * 8, cudaMemcpyDeviceToHost));
  return rc;
}

// Batched FP64 direct solve of `groups` (DIRECT systems) on stream st: one
// job per group in every kernel; the sequence is captured once into B's
// graph and replayed while the arguments, the RHS workspace and the set of
// modes stay the same.
static int direct_batched(sx_modal_s *s, DirectBatch &B, const std::vector<Group> &groups, double *d_u,
                          double *d_f, const double *d_bc, int nz, int plane_stride, cudaStream_t st) {
  for (auto &g : groups)
    if (s->sys[g.mode]->method != SX_DIRECT) {
      set_error("the batched band solve needs DIRECT systems (local mode %d is not)", g.mode);
      return SX_ERR_UNSUPPORTED;
    }
  int planes = 0;
  std::vector<int> modes;
  for (auto &g : groups) {
    planes += g.P;
    modes.push_back(g.mode);
  }
  SX_TRY(reserve_ws(*s, planes));
  const bool same = B.exec && B.key[0] == d_u && B.key[1] == d_f && B.key[2] == d_bc && B.key[3] == s->rhs.p &&
                    B.key[4] == s->Fb.p && B.key[5] == s->gess.p && B.nz == nz && B.stride == plane_stride &&
                    B.modes == modes;
  const MeshView M = s->mesh->view();
  if (!same || !s->use_graphs) {
    B.reset();
    const long long bcstride = (long long)std::max(s->mesh->nbound, 1) * s->mesh->np;
    std::vector<Job> jobs;
    int slot = 0;
    for (auto &g : groups) {
      jobs.push_back(make_job(*s, g, slot, d_u, d_f, d_bc, plane_stride, bcstride));
      slot += g.P;
    }
    if (B.djobs.n < jobs.size()) SX_TRY(B.djobs.alloc(jobs.size()));
    SX_CUDA(cudaMemcpyAsync(B.djobs.p, jobs.data(), jobs.size() * sizeof(Job), cudaMemcpyHostToDevice, st));
    SX_CUDA(cudaStreamSynchronize(st));
    SX_TRY(prepare_direct_kernels(M));
    B.sc = s->sched((int)jobs.size());
    B.jobs = jobs;
    B.modes = modes;
    if (!s->use_graphs) return direct_solve_jobs(M, B.djobs.p, jobs, st, B.sc, &B.launches);
    cudaGraph_t g = nullptr;
    SX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int rc = direct_solve_jobs(M, B.djobs.p, jobs, st, B.sc, &B.launches);
    const cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (rc != SX_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    SX_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(&B.exec, g, 0);
    cudaGraphDestroy(g);
    SX_CUDA(ie);
    B.key[0] = d_u;
    B.key[1] = d_f;
    B.key[2] = d_bc;
    B.key[3] = s->rhs.p;
    B.key[4] = s->Fb.p;
    B.key[5] = s->gess.p;
    B.nz = nz;
    B.stride = plane_stride;
  }
  SX_CUDA(cudaGraphLaunch(B.exec, st));
  return SX_OK;
}

int sx::cg_round_iters(double kratio, double hcon) {
  if (!(hcon > 0.0)) return CG_ROUND_CAP + 1;
  const double n = std::ceil(4.5 * std::sqrt(1.0 + kratio / hcon));
  return n > CG_ROUND_CAP ? CG_ROUND_CAP + 1 : (int)n;
}

bool sx::band_cheaper(int np, int nel, int nglobal, int nsolve, int nband, double kratio, double hcon,
                      int n_inner, double tol_rel, int max_refine, double reuse, double iter_floor_s,
                      double iter_factor) {
  const int per_round = std::max(std::max(n_inner, 1), cg_round_iters(kratio, hcon));
  if (per_round > CG_ROUND_CAP) return true;
  const int nn = np * np, next = 4 * (np - 1), nint = nn - next;
  const double rounds = std::max(1.0, std::ceil(-std::log10(std::max(tol_rel, 1e-15)) / 6.0));
  if (rounds > max_refine) return true;
  const double npts = nglobal + (double)nel * nint;
  const double iter_s = std::max(iter_floor_s, 2.0 * 4.0 * (8.0 * npts + 2.0 * (double)nel * nn) / 2.1e12);
  const double cg_s = rounds * per_round * iter_factor * iter_s;
  const double band_s =
      (2.0 * nsolve * (double)nband * 8.0 + (double)nel * ((double)next * nint + (double)nint * nint) * 8.0) /
      1.9e12;
  const double factor_s = reuse > 0.0 ? nsolve * (double)nband * nband / 3.9e12 / reuse : 0.0;
  return cg_s > band_s + factor_s;
}

// Route of a mode in the mixed-precision form: true = the FP64 band
// Cholesky (the mode must be factored), false = FP32 CG inside FP64
// refinement.
static bool route_direct(const sx_modal_s &s, const System &S, double tol_rel, int max_refine) {
  if (S.method != SX_DIRECT || !S.tiles.p) return false;
  if (s.mixed_route == 1) return false;
  if (s.mixed_route == 2) return true;
  const sx_mesh_s &M = *s.mesh;
  return band_cheaper(M.np, M.nel, M.nglobal, S.nsolve, M.nband, M.kratio, S.lambda2 + S.betak2, s.n_inner,
                      tol_rel, max_refine, 0.0);
}

// Mixed-precision batched form (sx_mixed.cu): the modes routed to the FP32
// iterations run as one FP32-CG / FP64-refinement solve of all their planes;
// the modes routed to the band Cholesky run as one batched FP64 direct solve
// on a second stream at the same time.
static int mixed_solve_batched(sx_modal s, double *d_u, double *d_f, const double *d_bc, int nz,
                               int plane_stride, double tol_rel, int max_refine, cudaStream_t st,
                               sx_solve_stats *stats) {
  std::vector<Group> groups;
  SX_TRY(plane_groups(*s, nz, groups));
  for (auto &u : s->uniq)
    if (!u->pcf.p) SX_TRY(system_build_jacobi_diag(*u, st));
  std::vector<Group> gd;
  std::vector<MxGroup> mg;
  std::vector<int> jmodes;
  for (auto &g : groups) {
    const System *S = s->sys[g.mode].get();
    if (route_direct(*s, *S, tol_rel, max_refine)) {
      gd.push_back(g);
    } else {
      mg.push_back({g.mode, g.plane0, g.P, S});
      jmodes.push_back(g.mode);
    }
  }
  int dplanes = 0;
  for (auto &g : gd) dplanes += g.P;
  if (!gd.empty()) {
    if (!s->aux) SX_CUDA(cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking));
    if (!s->ev_fork) SX_CUDA(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming));
    if (!s->ev_join) SX_CUDA(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming));
    SX_CUDA(cudaEventRecord(s->ev_fork, st));
    SX_CUDA(cudaStreamWaitEvent(s->aux, s->ev_fork, 0));
    SX_TRY(direct_batched(s, s->hyb, gd, d_u, d_f, d_bc, nz, plane_stride, s->aux));
    SX_CUDA(cudaEventRecord(s->ev_join, s->aux));
  }
  sx_solve_stats loc{};
  int rc = SX_OK;
  if (!mg.empty()) {
    // iterations per round: the knob, raised to what the worst-conditioned
    // mode needs for a 1e-6 cut per round (a restarted CG round that stops
    // short stalls the refinement)
    int n_inner = std::max(s->n_inner, 1), easiest = CG_ROUND_CAP;
    for (const MxGroup &g : mg) {
      const int need = std::min(CG_ROUND_CAP, cg_round_iters(s->mesh->kratio, g.sys->lambda2 + g.sys->betak2));
      n_inner = std::max(n_inner, need);
      easiest = std::min(easiest, need);
    }
    // stop flags pay when the easiest mode needs at most half the round
    const bool check_stop = 2 * easiest <= n_inner;
    const bool rebuild = !(s->mkey[0] == d_u && s->mkey[1] == d_f && s->mkey[2] == d_bc && s->mnz == nz &&
                           s->mstride == plane_stride && s->mixed.n_inner == n_inner && s->mmodes == jmodes &&
                           s->mixed.status == s->dstatus.p);
    s->mixed.status = s->dstatus.p;
    const MeshView M = s->mesh->view();
    rc = mixed_solve(M, s->mixed, mg, nz, s->num_modes, d_u, d_f, d_bc, plane_stride, rebuild, tol_rel,
                     max_refine, n_inner, check_stop, s->use_graphs, st, &loc);
    if (rc == SX_OK || rc == SX_WARN_STEP_LIMIT) {
      s->mkey[0] = d_u;
      s->mkey[1] = d_f;
      s->mkey[2] = d_bc;
      s->mnz = nz;
      s->mstride = plane_stride;
      s->mmodes = jmodes;
    }
  }
  if (!gd.empty()) SX_CUDA(cudaStreamWaitEvent(st, s->ev_join, 0));
  if (rc != SX_OK && rc != SX_WARN_STEP_LIMIT) return rc;
  if (stats) {
    *stats = loc;
    stats->planes_solved += dplanes;
    stats->planes_direct = dplanes;
    if (!gd.empty()) stats->kernel_launches += s->hyb.launches;
  }
  return rc;
}

namespace sx {

// Batched forms on stream st (no device-wide synchronisation).
int solve_batched_on(sx_modal_s *s, double *d_u, double *d_f, const double *d_bc, int nz, int plane_stride,
                     int precision, double tol_rel, int max_refine, cudaStream_t st, sx_solve_stats *stats) {
  if (precision == SX_MIXED_FP32)
    return mixed_solve_batched(s, d_u, d_f, d_bc, nz, plane_stride, tol_rel, max_refine, st, stats);
  std::vector<Group> groups;
  SX_TRY(plane_groups(*s, nz, groups));
  SX_TRY(direct_batched(s, s->fp64, groups, d_u, d_f, d_bc, nz, plane_stride, st));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    for (auto &g : groups) stats->planes_solved += g.P;
    stats->kernel_launches = s->fp64.launches;
  }
  return SX_OK;
}

}  // namespace sx

// Batched form: every mode's planes in each launch (one job per mode), the
// whole sequence captured once into a CUDA graph and replayed.
extern "C" int sx_field_solve_batched(sx_modal s, double *d_u, double *d_f, const double *d_bc, int nz,
                                      int plane_stride, int precision, double tol_rel, int max_refine,
                                      void *stream, sx_solve_stats *stats) {
  if (!s || !d_u || !d_f || plane_stride < s->mesh->nel * s->mesh->npnp) return SX_ERR_ARG;
  if (precision != SX_FP64 && precision != SX_MIXED_FP32) return SX_ERR_ARG;
  SX_TRY(check_mesh_device(*s->mesh, "sx_field_solve_batched"));
  if (!s->own) SX_CUDA(cudaStreamCreateWithFlags(&s->own, cudaStreamDefault));
  cudaStream_t st = stream ? (cudaStream_t)stream : s->own;
  const int rc = solve_batched_on(s, d_u, d_f, d_bc, nz, plane_stride, precision, tol_rel, max_refine, st,
                                  stats);
  if (rc != SX_OK && rc != SX_WARN_STEP_LIMIT) return rc;
  if (!stream) SX_TRY(take_status(s, true));
  return rc;
}

extern "C" int sx_modal_autotune(sx_modal s, double *d_u, const double *d_f, const double *d_bc, int nz,
                                 int plane_stride, int precision, double tol_rel, int max_refine, void *stream,
                                 sx_tune_result *out) {
  if (!s || !d_u || !d_f || plane_stride < s->mesh->nel * s->mesh->npnp) return SX_ERR_ARG;
  if (precision != SX_FP64 && precision != SX_MIXED_FP32) return SX_ERR_ARG;
  if (!s->own) SX_CUDA(cudaStreamCreateWithFlags(&s->own, cudaStreamDefault));
  cudaStream_t st = stream ? (cudaStream_t)stream : s->own;
  std::vector<Group> groups;
  SX_TRY(plane_groups(*s, nz, groups));
  // does this form run band sweeps, on how many systems, and how many tiles
  // do they stream per block column?
  int nj = precision == SX_FP64 ? (int)groups.size() : 0;
  if (precision != SX_FP64) {
    for (auto &u : s->uniq)
      if (!u->pcf.p) SX_TRY(system_build_jacobi_diag(*u, st));
    for (auto &g : groups) nj += route_direct(*s, *s->sys[g.mode], tol_rel, max_refine) ? 1 : 0;
  }
  const bool band = nj > 0;
  int J = 1;
  for (auto &u : s->uniq) J = std::max(J, u->J);
  // the occupancy queries below need the sweep kernels' shared-memory limit
  if (band) SX_TRY(prepare_direct_kernels(s->mesh->view()));
  const size_t n = (size_t)nz * plane_stride;
  DBuf<double> fw;  // the trials' forcing: a solve overwrites its forcing
  SX_TRY(fw.alloc(n));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  SX_CUDA(cudaEventCreate(&e0));
  SX_CUDA(cudaEventCreate(&e1));
  const int saved_cluster = s->forced_cluster, saved_stages = s->forced_stages, saved_lead = s->forced_lead;
  const int saved_inner = s->n_inner;
  struct Cand {
    BandSched sc;
    int inner;
  };
  Cand best{s->sched(std::max(nj, 1)), saved_inner};
  double best_t = INFINITY;
  bool best_ok = false;
  int trials = 0, rc = SX_OK;
  // one candidate: three solves (the first captures the graphs), the faster
  // of the last two; kept when it converges and beats the best so far
  auto trial = [&](const Cand &c) {
    s->forced_cluster = c.sc.C;
    s->forced_stages = c.sc.S;
    s->forced_lead = c.sc.Q;
    s->n_inner = c.inner;
    s->fp64.reset();  // the captured graphs bake in the schedule
    s->hyb.reset();
    double t_min = INFINITY;
    int r = SX_OK;
    for (int rep = 0; rep < 3 && (r == SX_OK || r == SX_WARN_STEP_LIMIT); rep++) {
      if (cudaMemcpyAsync(fw.p, d_f, n * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
        rc = SX_ERR_CUDA;
        return;
      }
      cudaEventRecord(e0, st);
      r = solve_batched_on(s, d_u, fw.p, d_bc, nz, plane_stride, precision, tol_rel, max_refine, st, nullptr);
      cudaEventRecord(e1, st);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        rc = SX_ERR_CUDA;
        return;
      }
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0) t_min = std::min(t_min, (double)ms);
    }
    if (r != SX_OK && r != SX_WARN_STEP_LIMIT) return;
    trials++;
    const bool ok = r == SX_OK;
    if ((ok && !best_ok) || (ok == best_ok && t_min < best_t)) {
      best_t = t_min;
      best_ok = ok;
      best = c;
    }
  };
  const int inner0 = precision == SX_MIXED_FP32 ? saved_inner : s->n_inner;
  if (band) {
    // (1) cluster size and ring depth, with the default leader share
    for (int S : {BAND_STAGES_MAX, 3, 2, 1})
      for (int C : {1, 2, 3, 4, 6, 8, 12, 16})
        if (rc == SX_OK && C <= J && band_active_clusters(C, 2, J + 2, S) > 0)
          trial({{C, S, default_lead(C, J)}, inner0});
    // (2) the leader's share on the best of those: none, or the last of every
    // K positions for K = C + 1, C + 2, 2C
    const BandSched b1 = best.sc;
    if (b1.C > 1)
      for (int K : {0, b1.C, b1.C + 1, b1.C + 2, 2 * b1.C})
        if (rc == SX_OK && K != b1.Q && (K == 0 || K <= J - 1) && (K != 2 * b1.C || 2 * b1.C > b1.C + 2))
          trial({{b1.C, b1.S, K}, inner0});
  }
  // (3) the floor on FP32 iterations per round, on the best band schedule
  if (precision == SX_MIXED_FP32) {
    const BandSched b2 = best.sc;
    for (int I : {8, 12, 16, 24})
      if (rc == SX_OK && I != inner0) trial({b2, I});
    if (rc == SX_OK && !band) trial({b2, inner0});
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // the graphs captured on the trial forcing must not outlive it
  s->fp64.reset();
  s->hyb.reset();
  s->mkey[0] = s->mkey[1] = s->mkey[2] = nullptr;
  s->sched_for.clear();
  if (trials) {
    // the choice is kept for this many systems per launch; hand-set band
    // knobs give way to it
    s->forced_cluster = s->forced_stages = 0;
    s->forced_lead = -1;
    if (band) s->sched_for[nj] = best.sc;
    s->n_inner = best.inner;
  } else {
    s->forced_cluster = saved_cluster;
    s->forced_stages = saved_stages;
    s->forced_lead = saved_lead;
    s->n_inner = saved_inner;
  }
  SX_CUDA(cudaStreamSynchronize(st));
  if (rc != SX_OK) return rc;
  if (!trials) {
    set_error("autotune: no candidate schedule solved");
    return SX_ERR_UNSUPPORTED;
  }
  if (out) {
    out->band_cluster = band ? best.sc.C : 0;
    out->band_stages = band ? best.sc.S : 0;
    out->band_lead = band ? best.sc.Q : 0;
    out->inner_iters = precision == SX_MIXED_FP32 ? s->n_inner : 0;
    out->ms = best_t;
    out->trials = trials;
  }
  return SX_OK;
}

sx_modal_s::HostPipe::~HostPipe() {
  views.clear();
  for (cudaEvent_t e : in) cudaEventDestroy(e);
  for (cudaEvent_t e : done) cudaEventDestroy(e);
  for (cudaStream_t x : cs) cudaStreamDestroy(x);
  if (h2d) cudaStreamDestroy(h2d);
  if (d2h) cudaStreamDestroy(d2h);
}

// Modes per chunk of the pipelined host entry.  When every mode is solved
// by the band Cholesky and there are 32 modes or more: eight chunks of at
// least 8 modes.  The chunks are solved side by side on their own streams,
// so their band sweeps share the GPU as one launch would, and small chunks
// shorten the ends of the pipeline: the last chunk's copy in and the copy
// out after it (config 3's 64 modes end to end: 38.0 ms with 8-mode chunks,
// 39.9 with 16, 43.2 with 32, 48.8 unpipelined, for a 31 ms solve).
// Otherwise half the modes, rounded up to a multiple of 16 (32 planes, one
// full lane chunk of the mixed form's FP32 kernels), at least 16.
constexpr int HOST_CHUNK_MIN = 16;
static int host_chunk_modes(int nmodes, bool all_band) {
  if (all_band && nmodes >= 32) return std::max(8, ((nmodes + 7) / 8 + 7) / 8 * 8);
  const int half = (nmodes + 1) / 2;
  return std::max(HOST_CHUNK_MIN, (half + HOST_CHUNK_MIN - 1) / HOST_CHUNK_MIN * HOST_CHUNK_MIN);
}

extern "C" int sx_field_solve_batched_host(sx_modal s, double *u, const double *f, const double *bc,
                                           int nz, int plane_stride, int precision, double tol_rel,
                                           int max_refine, sx_solve_stats *stats) {
  if (!s || !u || !f || nz <= 0 || plane_stride <= 0) return SX_ERR_ARG;
  SX_TRY(check_mesh_device(*s->mesh, "sx_field_solve_batched_host"));
  const size_t n = (size_t)nz * plane_stride;
  const size_t bcp = (size_t)std::max(s->mesh->nbound, 1) * s->mesh->np;  // bc values per plane
  const size_t nbc = (size_t)nz * bcp;
  if (s->hu.n < n) SX_TRY(s->hu.alloc(n));
  if (s->hf.n < n) SX_TRY(s->hf.alloc(n));
  if (bc && s->hbc.n < nbc) SX_TRY(s->hbc.alloc(nbc));
  if (!s->own) SX_CUDA(cudaStreamCreateWithFlags(&s->own, cudaStreamDefault));
  cudaStream_t st = s->own;
  const int nmodes = nz == 1 ? 1 : nz / 2;
  bool all_band = true;
  for (int l = 0; l < std::min(nmodes, s->num_modes) && all_band; l++) {
    const System &S = *s->sys[l];
    all_band = S.method == SX_DIRECT && S.tiles.p &&
               (precision == SX_FP64 || route_direct(*s, S, tol_rel, max_refine));
  }
  const int chunk = s->host_chunk > 0 ? s->host_chunk : host_chunk_modes(nmodes, all_band);
  const int nchunks = (nmodes + chunk - 1) / chunk;
  if (nchunks < 2 || nz % 2 || nmodes > s->num_modes) {
    SX_CUDA(cudaMemcpyAsync(s->hf.p, f, n * 8, cudaMemcpyHostToDevice, st));
    if (bc) SX_CUDA(cudaMemcpyAsync(s->hbc.p, bc, nbc * 8, cudaMemcpyHostToDevice, st));
    const int rc = solve_batched_on(s, s->hu.p, s->hf.p, bc ? s->hbc.p : nullptr, nz, plane_stride, precision,
                                    tol_rel, max_refine, st, stats);
    if (rc != SX_OK && rc != SX_WARN_STEP_LIMIT) return rc;
    SX_TRY(copy_solved_planes(u, s->hu.p, nz, plane_stride, s->base_mode, st));
    SX_TRY(take_status(s, true, st, false));
    return rc;
  }
  // Pipelined: every chunk's forcing goes up on one stream at once; each
  // chunk is solved on its own stream as soon as its copy has landed, so the
  // chunks' solves run side by side (with the band-sweep schedule of the
  // whole field, whose CTAs they share out between them), and a chunk's
  // solution goes down on a third stream as soon as it is solved.  Chunk c
  // covers modes [chunk c, chunk (c + 1)), planes [2 chunk c, 2 chunk (c + 1))
  // (chunk 0 keeps the Nyquist plane 1 in place).
  if (!s->pipe) s->pipe.reset(new sx_modal_s::HostPipe());
  sx_modal_s::HostPipe &P = *s->pipe;
  if (!P.h2d) SX_CUDA(cudaStreamCreateWithFlags(&P.h2d, cudaStreamNonBlocking));
  if (!P.d2h) SX_CUDA(cudaStreamCreateWithFlags(&P.d2h, cudaStreamNonBlocking));
  while ((int)P.in.size() < nchunks) {
    cudaEvent_t a = nullptr, b = nullptr;
    SX_CUDA(cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
    SX_CUDA(cudaEventCreateWithFlags(&b, cudaEventDisableTiming));
    P.in.push_back(a);
    P.done.push_back(b);
  }
  while ((int)P.views.size() < nchunks) P.views.emplace_back(new sx_modal_s());
  while ((int)P.cs.size() < nchunks) {
    cudaStream_t x = nullptr;
    SX_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
    P.cs.push_back(x);
  }
  // the schedule a launch over every mode would take (tuned or default)
  const BandSched psc = s->sched(nmodes);
  // the views share the system objects; their workspaces are their own
  SX_CUDA(cudaEventRecord(P.in[0], st));  // the device buffers are free once st's earlier work is done
  SX_CUDA(cudaStreamWaitEvent(P.h2d, P.in[0], 0));
  for (int c = 0; c < nchunks; c++) {
    const int m0 = c * chunk, m1 = std::min(nmodes, m0 + chunk);
    const size_t off = (size_t)2 * m0 * plane_stride, len = (size_t)2 * (m1 - m0) * plane_stride;
    SX_CUDA(cudaMemcpyAsync(s->hf.p + off, f + off, len * 8, cudaMemcpyHostToDevice, P.h2d));
    if (bc)
      SX_CUDA(cudaMemcpyAsync(s->hbc.p + 2 * m0 * bcp, bc + 2 * m0 * bcp, 2 * (m1 - m0) * bcp * 8,
                              cudaMemcpyHostToDevice, P.h2d));
    SX_CUDA(cudaEventRecord(P.in[c], P.h2d));
  }
  int rc = SX_OK;
  sx_solve_stats tot{};
  for (int c = 0; c < nchunks; c++) {
    const int m0 = c * chunk, m1 = std::min(nmodes, m0 + chunk);
    sx_modal_s &v = *P.views[c];
    const std::vector<std::shared_ptr<System>> sub(s->sys.begin() + m0, s->sys.begin() + m1);
    if (v.mesh != s->mesh || v.base_mode != s->base_mode + m0 || v.num_modes != m1 - m0 || v.sys != sub)
      v.rebind(s->mesh, s->base_mode + m0, m1 - m0, s->method, sub);
    cudaStream_t vs = P.cs[c];
    v.own = vs;
    v.own_stream_external = true;
    v.n_inner = s->n_inner;
    v.mixed_route = s->mixed_route;
    if (v.forced_cluster != psc.C || v.forced_stages != psc.S || v.forced_lead != psc.Q) {
      v.forced_cluster = psc.C;
      v.forced_stages = psc.S;
      v.forced_lead = psc.Q;
      v.fp64.reset();
      v.hyb.reset();
    }
    if (!v.dstatus.p) {
      SX_TRY(v.dstatus.alloc(1));
      SX_TRY(v.dstatus.zero(vs));
    }
    const size_t off = (size_t)2 * m0 * plane_stride;
    SX_CUDA(cudaStreamWaitEvent(vs, P.in[c], 0));
    sx_solve_stats cs{};
    const int r = solve_batched_on(&v, s->hu.p + off, s->hf.p + off, bc ? s->hbc.p + 2 * m0 * bcp : nullptr,
                                   2 * (m1 - m0), plane_stride, precision, tol_rel, max_refine, vs, &cs);
    if (r != SX_OK && r != SX_WARN_STEP_LIMIT) return r;
    if (r == SX_WARN_STEP_LIMIT) rc = r;
    SX_CUDA(cudaEventRecord(P.done[c], vs));
    SX_CUDA(cudaStreamWaitEvent(st, P.done[c], 0));  // later work on st follows every chunk
    SX_CUDA(cudaStreamWaitEvent(P.d2h, P.done[c], 0));
    SX_TRY(copy_solved_planes(u + off, s->hu.p + off, 2 * (m1 - m0), plane_stride, v.base_mode, P.d2h));
    tot.planes_solved += cs.planes_solved;
    tot.planes_direct += cs.planes_direct;
    tot.iterations_max = std::max(tot.iterations_max, cs.iterations_max);
    tot.iterations_total += cs.iterations_total;
    tot.refinements = std::max(tot.refinements, cs.refinements);
    tot.final_rel_residual = std::max(tot.final_rel_residual, cs.final_rel_residual);
    tot.kernel_launches += cs.kernel_launches;
  }
  SX_CUDA(cudaStreamSynchronize(P.d2h));
  for (int c = 0; c < (int)P.views.size(); c++)
    if (P.views[c]->dstatus.p) SX_TRY(take_status(P.views[c].get(), true, P.cs[c], false));
  if (stats) *stats = tot;
  return rc;
}

int sx::check_mesh_device(const sx_mesh_s &M, const char *who) {
  int dev = -1;
  SX_CUDA(cudaGetDevice(&dev));
  if (dev != M.device) {
    set_error("%s: the current device is %d, but the mesh and its systems live on device %d", who, dev, M.device);
    return SX_ERR_ARG;
  }
  return SX_OK;
}

int sx::copy_solved_planes(double *h_u, const double *d_u, int nz, int plane_stride, int base_mode,
                           cudaStream_t st) {
  const size_t ps = (size_t)plane_stride;
  if (nz > 1 && base_mode == 0) {
    SX_CUDA(cudaMemcpyAsync(h_u, d_u, ps * 8, cudaMemcpyDeviceToHost, st));
    if (nz > 2)
      SX_CUDA(cudaMemcpyAsync(h_u + 2 * ps, d_u + 2 * ps, (size_t)(nz - 2) * ps * 8, cudaMemcpyDeviceToHost,
                              st));
  } else {
    SX_CUDA(cudaMemcpyAsync(h_u, d_u, (size_t)nz * ps * 8, cudaMemcpyDeviceToHost, st));
  }
  return SX_OK;
}

extern "C" int sx_profile_band_sweeps(sx_modal s, int reps, void *stream) {
  if (!s || reps <= 0 || s->fp64.jobs.empty()) return SX_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  for (int r = 0; r < reps; r++)
    SX_TRY(band_sweep_jobs(s->fp64.djobs.p, s->fp64.jobs, s->fp64.sc, st));
  return SX_OK;
}

extern "C" int sx_profile_mixed_iterations(sx_modal s, int reps, void *stream) {
  if (!s) return SX_ERR_ARG;
  return mixed_profile_iterations(s->mesh->view(), s->mixed, reps, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// multi-mesh batch
// ---------------------------------------------------------------------------

sx_batch_s::~sx_batch_s() {
  if (dexec) cudaGraphExecDestroy(dexec);
  if (ev_fork) cudaEventDestroy(ev_fork);
  if (ev_join) cudaEventDestroy(ev_join);
  if (aux) cudaStreamDestroy(aux);
  if (own) cudaStreamDestroy(own);
}

extern "C" int sx_batch_create(sx_batch *out) {
  if (!out) return SX_ERR_ARG;
  *out = new sx_batch_s();
  return SX_OK;
}

extern "C" int sx_batch_destroy(sx_batch b) {
  delete b;
  return SX_OK;
}

namespace {

// One member's share of a batch solve.
struct Part {
  sx_modal s = nullptr;
  std::vector<Group> gd;       // plane groups for the band Cholesky
  std::vector<MxGroup> mg;     // plane groups for the FP32 iterations
  std::vector<int> jmodes;     // local modes of mg
  double *u = nullptr, *f = nullptr;
  const double *bc = nullptr;
  int nz = 0, stride = 0;
};

void key_ptr(std::vector<long long> &k, const void *p) { k.push_back((long long)(intptr_t)p); }

}  // namespace

// The band Cholesky part of a batch: per member its RHS kernels, then one
// band-sweep launch over every member's jobs, then per member the interior
// back-substitution; captured once per member set and buffers.
static int batch_direct(sx_batch b, std::vector<Part> &parts, bool graphs, cudaStream_t st) {
  std::vector<long long> key;
  for (Part &q : parts) {
    if (q.gd.empty()) continue;
    int planes = 0;
    for (auto &g : q.gd) planes += g.P;
    SX_TRY(reserve_ws(*q.s, planes));
    key_ptr(key, q.s);
    key_ptr(key, q.u);
    key_ptr(key, q.f);
    key_ptr(key, q.bc);
    key_ptr(key, q.s->rhs.p);
    key_ptr(key, q.s->Fb.p);
    key_ptr(key, q.s->gess.p);
    key.push_back(q.nz);
    key.push_back(q.stride);
    key.push_back(q.s->forced_cluster);
    key.push_back(q.s->forced_stages);
    key.push_back(q.s->forced_lead);
    for (auto &g : q.gd) key.push_back(g.mode);
    key.push_back(-1);
  }
  if (key.empty()) return SX_OK;
  if (b->dexec && graphs && key == b->dkey) {
    SX_CUDA(cudaGraphLaunch(b->dexec, st));
    return SX_OK;
  }
  if (b->dexec) cudaGraphExecDestroy(b->dexec);
  b->dexec = nullptr;
  b->dkey.clear();
  std::vector<Job> jobs;
  std::vector<size_t> j0;
  int maxJ = 1, maxP = 1, forced = 0, fstages = 0, flead = -1;
  for (Part &q : parts) {
    j0.push_back(jobs.size());
    if (q.gd.empty()) continue;
    const long long bcstride = (long long)std::max(q.s->mesh->nbound, 1) * q.s->mesh->np;
    int slot = 0;
    for (auto &g : q.gd) {
      jobs.push_back(make_job(*q.s, g, slot, q.u, q.f, q.bc, q.stride, bcstride));
      maxJ = std::max(maxJ, jobs.back().J);
      maxP = std::max(maxP, g.P);
      slot += g.P;
    }
    forced = std::max(forced, q.s->forced_cluster);
    fstages = std::max(fstages, q.s->forced_stages);
    flead = std::max(flead, q.s->forced_lead);
    SX_TRY(prepare_direct_kernels(q.s->mesh->view()));
  }
  j0.push_back(jobs.size());
  if (b->djobs.n < jobs.size()) SX_TRY(b->djobs.alloc(jobs.size()));
  SX_CUDA(cudaMemcpyAsync(b->djobs.p, jobs.data(), jobs.size() * sizeof(Job), cudaMemcpyHostToDevice, st));
  SX_CUDA(cudaStreamSynchronize(st));
  b->jobs = jobs;
  b->sc = BandSched();
  b->sc.C = forced > 0 ? forced
                       : pick_cluster((int)jobs.size(), std::min(16, std::max(1, maxJ)), maxP <= 2 ? 2 : 8,
                                      maxJ + 2, &b->sc.S, fstages);
  if (forced > 0 && fstages > 0) b->sc.S = fstages;
  b->sc.Q = flead >= 0 ? flead : default_lead(b->sc.C, maxJ);
  auto body = [&]() -> int {
    int nl = 0;
    for (size_t i = 0; i < parts.size(); i++) {
      if (parts[i].gd.empty()) continue;
      const std::vector<Job> slice(jobs.begin() + j0[i], jobs.begin() + j0[i + 1]);
      SX_TRY(direct_rhs_jobs(parts[i].s->mesh->view(), b->djobs.p + j0[i], slice, st, &nl));
    }
    SX_TRY(band_sweep_jobs(b->djobs.p, jobs, b->sc, st));
    nl++;
    for (size_t i = 0; i < parts.size(); i++) {
      if (parts[i].gd.empty()) continue;
      SX_TRY(direct_backsub_jobs(parts[i].s->mesh->view(), b->djobs.p + j0[i], (int)(j0[i + 1] - j0[i]), st,
                                 &nl));
    }
    b->dlaunches = nl;
    return SX_OK;
  };
  if (!graphs) return body();
  cudaGraph_t g = nullptr;
  SX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  const int rc = body();
  const cudaError_t ce = cudaStreamEndCapture(st, &g);
  if (rc != SX_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  SX_CUDA(ce);
  const cudaError_t ie = cudaGraphInstantiate(&b->dexec, g, 0);
  cudaGraphDestroy(g);
  SX_CUDA(ie);
  b->dkey = key;
  SX_CUDA(cudaGraphLaunch(b->dexec, st));
  return SX_OK;
}

extern "C" int sx_batch_solve(sx_batch b, int count, const sx_modal *modals, double *const *d_u,
                              double *const *d_f, const double *const *d_bc, const int *nz, const int *plane_stride,
                              int precision, double tol_rel, int max_refine, void *stream, sx_solve_stats *stats) {
  if (!b || count <= 0 || !modals || !d_u || !d_f || !nz || !plane_stride) return SX_ERR_ARG;
  if (precision != SX_FP64 && precision != SX_MIXED_FP32) return SX_ERR_ARG;
  std::vector<Part> parts(count);
  for (int i = 0; i < count; i++) {
    sx_modal s = modals[i];
    if (!s || !d_u[i] || !d_f[i] || plane_stride[i] < s->mesh->nel * s->mesh->npnp) return SX_ERR_ARG;
    for (int j = 0; j < i; j++)
      if (modals[j] == s) {
        set_error("sx_batch_solve: modal system %d appears twice (members %d and %d)", i, j, i);
        return SX_ERR_ARG;
      }
    Part &q = parts[i];
    q.s = s;
    q.u = d_u[i];
    q.f = d_f[i];
    q.bc = d_bc ? d_bc[i] : nullptr;
    q.nz = nz[i];
    q.stride = plane_stride[i];
  }
  if (!b->own) SX_CUDA(cudaStreamCreateWithFlags(&b->own, cudaStreamDefault));
  cudaStream_t st = stream ? (cudaStream_t)stream : b->own;
  // plane groups and their routes
  bool any_direct = false, any_mixed = false;
  for (Part &q : parts) {
    std::vector<Group> groups;
    SX_TRY(plane_groups(*q.s, q.nz, groups));
    if (!q.s->dstatus.p) {
      SX_TRY(q.s->dstatus.alloc(1));
      SX_TRY(q.s->dstatus.zero(st));
    }
    if (precision == SX_FP64) {
      for (auto &g : groups)
        if (q.s->sys[g.mode]->method != SX_DIRECT) {
          set_error("the batched band solve needs DIRECT systems (local mode %d is not)", g.mode);
          return SX_ERR_UNSUPPORTED;
        }
      q.gd = groups;
    } else {
      for (auto &u : q.s->uniq)
        if (!u->pcf.p) SX_TRY(system_build_jacobi_diag(*u, st));
      for (auto &g : groups) {
        const System *S = q.s->sys[g.mode].get();
        if (route_direct(*q.s, *S, tol_rel, max_refine)) {
          q.gd.push_back(g);
        } else {
          q.mg.push_back({g.mode, g.plane0, g.P, S});
          q.jmodes.push_back(g.mode);
        }
      }
    }
    any_direct |= !q.gd.empty();
    any_mixed |= !q.mg.empty();
  }
  const bool graphs = b->use_graphs;
  cudaStream_t sd = st;  // stream of the band part
  if (any_direct && any_mixed) {
    if (!b->aux) SX_CUDA(cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking));
    if (!b->ev_fork) SX_CUDA(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
    if (!b->ev_join) SX_CUDA(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
    SX_CUDA(cudaEventRecord(b->ev_fork, st));
    SX_CUDA(cudaStreamWaitEvent(b->aux, b->ev_fork, 0));
    sd = b->aux;
  }
  if (any_direct) SX_TRY(batch_direct(b, parts, graphs, sd));
  if (any_direct && any_mixed) SX_CUDA(cudaEventRecord(b->ev_join, b->aux));
  int rc = SX_OK;
  std::vector<MxItem> items;
  std::vector<int> item_of(count, -1);
  if (any_mixed) {
    std::vector<long long> key;
    int n_inner = 1, easiest = CG_ROUND_CAP;
    for (int i = 0; i < count; i++) {
      Part &q = parts[i];
      if (q.mg.empty()) continue;
      n_inner = std::max(n_inner, std::max(q.s->n_inner, 1));
      for (const MxGroup &g : q.mg) {
        const int need =
            std::min(CG_ROUND_CAP, cg_round_iters(q.s->mesh->kratio, g.sys->lambda2 + g.sys->betak2));
        n_inner = std::max(n_inner, need);
        easiest = std::min(easiest, need);
      }
      q.s->mixed.status = q.s->dstatus.p;
      MxItem it;
      it.M = q.s->mesh->view();
      it.W = &q.s->mixed;
      it.groups = q.mg;
      it.nz = q.nz;
      it.num_modes = q.s->num_modes;
      it.u = q.u;
      it.f = q.f;
      it.bc = q.bc;
      it.stride = q.stride;
      item_of[i] = (int)items.size();
      items.push_back(it);
      key_ptr(key, q.s);
      key_ptr(key, q.u);
      key_ptr(key, q.f);
      key_ptr(key, q.bc);
      key_ptr(key, q.s->dstatus.p);
      key.push_back(q.nz);
      key.push_back(q.stride);
      for (int m : q.jmodes) key.push_back(m);
      key.push_back(-1);
    }
    key.push_back(n_inner);
    const bool rebuild = key != b->mkey;
    const bool check_stop = 2 * easiest <= n_inner;
    rc = mixed_solve_multi(items, b->mixed, rebuild, tol_rel, max_refine, n_inner, check_stop, graphs, st);
    if (rc == SX_OK || rc == SX_WARN_STEP_LIMIT)
      b->mkey = key;
    else
      b->mkey.clear();
  }
  if (any_direct && any_mixed) SX_CUDA(cudaStreamWaitEvent(st, b->ev_join, 0));
  if (rc != SX_OK && rc != SX_WARN_STEP_LIMIT) return rc;
  if (stats) {
    for (int i = 0; i < count; i++) {
      sx_solve_stats &S = stats[i];
      if (item_of[i] >= 0)
        S = items[item_of[i]].stats;
      else
        std::memset(&S, 0, sizeof(S));
      int dplanes = 0;
      for (auto &g : parts[i].gd) dplanes += g.P;
      S.planes_solved += dplanes;
      S.planes_direct = dplanes;
      if (dplanes) S.kernel_launches += b->dlaunches;
    }
  }
  if (!stream)
    for (Part &q : parts) SX_TRY(take_status(q.s, true, st, false));
  return rc;
}
