// sx_serve.cu -- continuous-batching request loop for Helmholtz solves.
//
// Requests (a mesh, per-mode Helmholtz constants, forcing planes) are queued
// by sx_server_submit and served by `slots` worker threads, each owning a
// non-blocking CUDA stream, a multi-mesh batch object and a pool of
// per-request workspaces.  A free worker takes every admissible pending
// request, in arrival order and up to max_batch, builds what the cache does
// not hold (element geometry, per-mode systems, one batched factorisation
// for the batch's new band factors) and solves the requests together with
// sx_batch_solve: one launch per kernel and element order covers all of
// them.  Requests that arrive while batches are on the device join the next
// one.  Admission is bounded by a device-memory budget: a request is
// admitted when the cached objects plus the reservations of the requests in
// flight plus its own estimate fit; least-recently-used cache entries no
// request is using are evicted to make room.  Element geometry (per mesh)
// and per-mode systems (Jacobi diagonals, or factored condensed matrices)
// stay resident across requests, keyed by (mesh contents, lambda2, betak2,
// kind), as the reference's MatrixSys cache keys them (src/matrix.cpp:85-102,
// 326-347).  A request's result is the same alone or in a batch within the
// solve tolerance: the batch shares the iteration count per refinement round
// and the number of rounds, each plane's arithmetic is its own.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "sx_modal.h"

using namespace sx;
using Clock = std::chrono::steady_clock;

namespace {

uint64_t fnv(uint64_t h, const void *p, size_t n) {
  const unsigned char *c = static_cast<const unsigned char *>(p);
  for (size_t i = 0; i < n; i++) {
    h ^= c[i];
    h *= 1099511628211ull;
  }
  return h;
}

struct MeshCopy {
  int np = 0, nel = 0, nglobal = 0, nsolve = 0, nband = 0, nbound = 0;
  double kratio = 0.0;  // stiffness / mass diagonal ratio (routes the mixed form)
  std::vector<double> x, y, bK, bC;
  std::vector<int> btog, bmask, be, bs, bk;
  uint64_t key = 0;
  sx_mesh_desc desc() const {
    sx_mesh_desc d;
    d.np = np; d.nel = nel; d.x = x.data(); d.y = y.data();
    d.btog = btog.data(); d.bmask = bmask.data();
    d.nglobal = nglobal; d.nsolve = nsolve; d.nband = nband; d.nbound = nbound;
    d.b_elmt = be.data(); d.b_side = bs.data(); d.b_kind = bk.data();
    d.b_K = bK.data(); d.b_C = bC.data();
    return d;
  }
};

struct Req {
  uint64_t id = 0;
  MeshCopy mesh;
  int base_mode = 0, num_modes = 0, nz = 0, stride = 0;
  std::vector<double> lam, bk2, f, bc;
  std::vector<int> kinds;  // per mode: system kind, fixed when admitted
  double *u = nullptr;
  Clock::time_point t_submit;
  size_t reserve = 0;  // bytes reserved while in flight
  bool done = false;
  int status = SX_OK;
  double latency_ms = 0.0;
};

struct MeshEntry {
  std::unique_ptr<sx_mesh_s> mesh;
  size_t bytes = 0;
  int refs = 0;
  uint64_t last_use = 0;
};

struct SysEntry {
  std::shared_ptr<System> sys;
  uint64_t mesh_key = 0;
  size_t bytes = 0;
  int refs = 0;
  uint64_t last_use = 0;
};

size_t mesh_estimate(const MeshCopy &m) {
  const size_t nn = (size_t)m.np * m.np, next = 4 * (m.np - 1);
  return (size_t)m.nel * nn * (5 * 8 + 4 * 4 + 16 + 1) + (size_t)m.nel * next * (4 * 3 + 16) +
         (size_t)m.nglobal * 32 +
         (size_t)m.nbound * m.np * 8 + 4096;
}

size_t system_estimate(const MeshCopy &m, int kind) {
  const size_t nn = (size_t)m.np * m.np, next = 4 * (m.np - 1), nint = nn - next;
  const size_t npts = m.nglobal + (size_t)m.nel * nint;
  size_t b = npts * 12;  // Jacobi diagonal, FP64 + FP32
  if (kind == SX_DIRECT) {
    const size_t nblk = (m.nsolve + NB - 1) / NB, J = (m.nband - 1 + NB - 1) / NB;
    b += (nblk * (J + 2)) * TSZ * 8 + (size_t)m.nel * (next * nint + nint * nint) * 8;
  }
  return b;
}

size_t work_estimate(const MeshCopy &m, int nz, int precision) {
  const size_t nn = (size_t)m.np * m.np, next = 4 * (m.np - 1), nint = nn - next;
  const size_t npts = m.nglobal + (size_t)m.nel * nint;
  const size_t PP = ((nz + MX_CH - 1) / MX_CH) * MX_CH;
  size_t b = 2 * (size_t)nz * m.nel * nn * 8 + (size_t)nz * std::max(m.nbound, 1) * m.np * 8;  // I/O
  if (precision == SX_MIXED_FP32)
    b += PP * npts * (2 * 8 + 9 * 4) + PP * m.nel * nn * 8 + 2 * PP * m.nel * next * 4 + PP * m.nglobal * 8 +
         npts * (nz / 2 + 1) * 4;
  else
    b += (size_t)nz * ((m.nsolve + NB) * 8 + (size_t)m.nel * next * 8 + (size_t)m.nglobal * 8);
  return b;
}

}  // namespace

struct sx_server_s {
  sx_server_config cfg{};
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req *> pending;
  std::unordered_map<uint64_t, std::unique_ptr<Req>> reqs;
  uint64_t next_id = 1, tick = 0;
  bool stopping = false;
  int inflight = 0;
  size_t bytes_cached = 0, bytes_reserved = 0;
  std::unordered_map<uint64_t, MeshEntry> meshes;
  std::map<std::tuple<uint64_t, uint64_t, uint64_t, int>, SysEntry> systems;
  std::mutex build_mu;  // serialises construction of cache entries
  std::vector<std::thread> workers;
  std::vector<double> latencies;
  sx_server_stats st{};

  // System kind of one mode (caller holds mu): SX_DIRECT for SX_FP64.  For
  // SX_MIXED_FP32 a cached factor is used when there is one; otherwise the
  // mode is factored only when the band Cholesky, with its factorisation
  // charged to this request alone, beats the FP32 iterations (or when those
  // would not converge within max_refine rounds).
  int mode_kind(const MeshCopy &m, double lam, double bk2) const {
    if (cfg.precision == SX_FP64) return SX_DIRECT;
    uint64_t a, b;
    std::memcpy(&a, &lam, 8);
    std::memcpy(&b, &bk2, 8);
    if (systems.count(std::make_tuple(m.key, a, b, (int)SX_DIRECT))) return SX_DIRECT;
    return band_cheaper(m.np, m.nel, m.nglobal, m.nsolve, m.nband, m.kratio, lam + bk2, cfg.inner_iters,
                        cfg.tol_rel, cfg.max_refine, 1.0)
               ? SX_DIRECT
               : SX_JACPCG;
  }
  bool admissible(Req *r, size_t &need);
  void evict_for(size_t need, uint64_t keep_mesh);
  void worker(int slot);
  // One request's mesh and systems, looked up or built (caller holds
  // build_mu); new band factors are appended to to_factor.
  struct Prep {
    sx_mesh_s *mesh = nullptr;
    std::vector<std::shared_ptr<System>> sys;
    std::vector<std::tuple<uint64_t, uint64_t, uint64_t, int>> keys;
    bool mesh_ref = false;
  };
  int prepare(Req *r, Prep &p, std::vector<System *> &to_factor, cudaStream_t stream);
  void release(const Req *r, const Prep &p);
  // A worker's workspace for one batch member.
  struct Member {
    std::unique_ptr<sx_modal_s> ws;
    DBuf<double> du, df, dbc;
    size_t bytes = 0;  // estimate of what the last request left allocated
  };
  void serve_batch(std::vector<Req *> &batch, std::vector<std::unique_ptr<Member>> &pool, sx_batch b,
                   cudaStream_t stream);
};

// Memory this request still needs beyond what is cached (caller holds mu).
bool sx_server_s::admissible(Req *r, size_t &need) {
  need = work_estimate(r->mesh, r->nz, cfg.precision);
  if (!meshes.count(r->mesh.key)) need += mesh_estimate(r->mesh);
  r->kinds.resize(r->num_modes);
  for (int l = 0; l < r->num_modes; l++) {
    const int kind = r->kinds[l] = mode_kind(r->mesh, r->lam[l], r->bk2[l]);
    uint64_t a, b;
    std::memcpy(&a, &r->lam[l], 8);
    std::memcpy(&b, &r->bk2[l], 8);
    if (!systems.count(std::make_tuple(r->mesh.key, a, b, kind))) need += system_estimate(r->mesh, kind);
  }
  return bytes_cached + bytes_reserved + need <= cfg.hbm_budget;
}

// Evict least-recently-used unreferenced entries until `need` fits
// (caller holds mu).
void sx_server_s::evict_for(size_t need, uint64_t keep_mesh) {
  while (bytes_cached + bytes_reserved + need > cfg.hbm_budget) {
    // systems first (cheaper to rebuild for Jacobi; factors are the big ones)
    auto sv = systems.end();
    for (auto it = systems.begin(); it != systems.end(); ++it)
      if (it->second.refs == 0 && (sv == systems.end() || it->second.last_use < sv->second.last_use)) sv = it;
    if (sv != systems.end()) {
      bytes_cached -= sv->second.bytes;
      systems.erase(sv);
      st.evictions++;
      continue;
    }
    auto mv = meshes.end();
    for (auto it = meshes.begin(); it != meshes.end(); ++it) {
      if (it->second.refs != 0 || it->first == keep_mesh) continue;
      bool used = false;
      for (auto &s : systems)
        if (s.second.mesh_key == it->first) used = true;
      if (!used && (mv == meshes.end() || it->second.last_use < mv->second.last_use)) mv = it;
    }
    if (mv == meshes.end()) return;
    bytes_cached -= mv->second.bytes;
    meshes.erase(mv);
    st.evictions++;
  }
}

int sx_server_s::prepare(Req *r, Prep &pp, std::vector<System *> &to_factor, cudaStream_t stream) {
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = meshes.find(r->mesh.key);
    if (it != meshes.end()) {
      pp.mesh = it->second.mesh.get();
      it->second.refs++;
      it->second.last_use = ++tick;
      pp.mesh_ref = true;
      st.mesh_hits++;
    }
  }
  if (!pp.mesh) {
    const sx_mesh_desc d = r->mesh.desc();
    sx_mesh m = nullptr;
    SX_TRY(sx_mesh_create(&d, &m));
    std::lock_guard<std::mutex> lk(mu);
    MeshEntry &e = meshes[r->mesh.key];
    e.mesh.reset(m);
    e.bytes = mesh_estimate(r->mesh);
    e.refs = 1;
    e.last_use = ++tick;
    bytes_cached += e.bytes;
    pp.mesh = m;
    pp.mesh_ref = true;
    st.mesh_misses++;
  }
  pp.sys.resize(r->num_modes);
  for (int l = 0; l < r->num_modes; l++) {
    const int kind = r->kinds[l];
    uint64_t a, b;
    std::memcpy(&a, &r->lam[l], 8);
    std::memcpy(&b, &r->bk2[l], 8);
    const auto key = std::make_tuple(r->mesh.key, a, b, kind);
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = systems.find(key);
      if (it != systems.end()) {
        pp.sys[l] = it->second.sys;
        it->second.refs++;
        it->second.last_use = ++tick;
        pp.keys.push_back(key);
        st.system_hits++;
        continue;
      }
    }
    auto S = std::make_shared<System>();
    S->mesh = pp.mesh;
    S->lambda2 = r->lam[l];
    S->betak2 = r->bk2[l];
    S->method = kind;
    if (kind == SX_DIRECT) {
      SX_TRY(system_build_direct(*S, stream));
      if (S->nsolve > 0) to_factor.push_back(S.get());
      SX_TRY(system_build_jacobi_diag(*S, stream));
    } else {
      SX_TRY(system_build_jacobi(*S, stream));
    }
    pp.sys[l] = S;
    std::lock_guard<std::mutex> lk(mu);
    SysEntry &e = systems[key];
    e.sys = S;
    e.mesh_key = r->mesh.key;
    e.bytes = system_estimate(r->mesh, kind);
    e.refs = 1;
    e.last_use = ++tick;
    bytes_cached += e.bytes;
    pp.keys.push_back(key);
    st.system_misses++;
  }
  return SX_OK;
}

void sx_server_s::release(const Req *r, const Prep &pp) {
  std::lock_guard<std::mutex> lk(mu);
  if (pp.mesh_ref) {
    auto mi = meshes.find(r->mesh.key);
    if (mi != meshes.end()) mi->second.refs--;
  }
  for (auto &k : pp.keys) {
    auto si = systems.find(k);
    if (si != systems.end()) si->second.refs--;
  }
}

// Workspaces above this size are freed after their batch instead of kept
// for the next one (a pool slot otherwise holds the largest request it saw).
constexpr size_t KEEP_WS_BYTES = size_t(256) << 20;

void sx_server_s::serve_batch(std::vector<Req *> &batch, std::vector<std::unique_ptr<Member>> &pool, sx_batch b,
                              cudaStream_t stream) {
  const int n = (int)batch.size();
  const auto t0 = Clock::now();
  std::vector<Prep> prep(n);
  std::vector<int> rc(n, SX_OK);
  {
    // look up or build the meshes and systems (one builder at a time), then
    // factor the batch's new band systems together
    std::lock_guard<std::mutex> bl(build_mu);
    std::vector<System *> to_factor;
    for (int i = 0; i < n; i++) rc[i] = prepare(batch[i], prep[i], to_factor, stream);
    const int fr = factor_batch(to_factor, stream);
    if (fr != SX_OK)
      for (int i = 0; i < n; i++) rc[i] = rc[i] == SX_OK ? fr : rc[i];
  }
  const auto t1 = Clock::now();
  while ((int)pool.size() < n) pool.emplace_back(new Member());
  std::vector<sx_modal> mods;
  std::vector<double *> du, df;
  std::vector<const double *> dbc;
  std::vector<int> nz, stride, idx;
  bool any_bc = false;
  for (int i = 0; i < n; i++) {
    if (rc[i] != SX_OK) continue;
    Req *r = batch[i];
    Member &m = *pool[i];
    if (!m.ws) {
      m.ws.reset(new sx_modal_s());
      m.ws->own = stream;
      m.ws->own_stream_external = true;
      m.ws->use_graphs = false;
    }
    sx_modal_s &ws = *m.ws;
    ws.rebind(prep[i].mesh, r->base_mode, r->num_modes, cfg.precision == SX_FP64 ? SX_DIRECT : SX_MIXED,
              prep[i].sys);
    ws.n_inner = cfg.inner_iters;
    const size_t len = (size_t)r->nz * r->stride;
    int e = SX_OK;
    if (m.du.n < len) e = m.du.alloc(len);
    if (e == SX_OK && m.df.n < len) e = m.df.alloc(len);
    if (e == SX_OK && !r->bc.empty() && m.dbc.n < r->bc.size()) e = m.dbc.alloc(r->bc.size());
    if (e == SX_OK && cudaMemcpyAsync(m.df.p, r->f.data(), len * 8, cudaMemcpyHostToDevice, stream) != cudaSuccess)
      e = SX_ERR_CUDA;
    if (e == SX_OK && !r->bc.empty() &&
        cudaMemcpyAsync(m.dbc.p, r->bc.data(), r->bc.size() * 8, cudaMemcpyHostToDevice, stream) != cudaSuccess)
      e = SX_ERR_CUDA;
    if (e != SX_OK) {
      rc[i] = e;
      continue;
    }
    m.bytes = work_estimate(r->mesh, r->nz, cfg.precision);
    mods.push_back(&ws);
    du.push_back(m.du.p);
    df.push_back(m.df.p);
    dbc.push_back(r->bc.empty() ? nullptr : m.dbc.p);
    any_bc |= !r->bc.empty();
    nz.push_back(r->nz);
    stride.push_back(r->stride);
    idx.push_back(i);
  }
  if (!mods.empty()) {
    std::vector<sx_solve_stats> sst(mods.size());
    int br = sx_batch_solve(b, (int)mods.size(), mods.data(), du.data(), df.data(), any_bc ? dbc.data() : nullptr,
                            nz.data(), stride.data(), cfg.precision, cfg.tol_rel, cfg.max_refine, stream,
                            sst.data());
    for (size_t k = 0; k < idx.size(); k++) {
      const int i = idx[k];
      Req *r = batch[i];
      int c = br;
      if (br == SX_OK || br == SX_WARN_STEP_LIMIT) {
        c = copy_solved_planes(r->u, du[k], r->nz, r->stride, r->base_mode, stream);
        if (c == SX_OK)
          c = (cfg.precision == SX_MIXED_FP32 && !(sst[k].final_rel_residual <= cfg.tol_rel)) ? SX_WARN_STEP_LIMIT
                                                                                             : SX_OK;
      }
      rc[i] = c;
    }
    if (cudaStreamSynchronize(stream) != cudaSuccess) {
      set_error("serving: batch solve or device -> host copy failed");
      for (int i : idx) rc[i] = SX_ERR_CUDA;
    }
    // the batch's device-side status words (bounded waits that ran out)
    for (size_t k = 0; k < idx.size(); k++) {
      int h = 0;
      sx_modal_s &ws = *pool[idx[k]]->ws;
      if (ws.dstatus.p && cudaMemcpy(&h, ws.dstatus.p, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess && h) {
        cudaMemset(ws.dstatus.p, 0, sizeof(int));
        rc[idx[k]] = SX_ERR_TIMEOUT;
      }
    }
  }
  const auto t2 = Clock::now();
  for (int i = 0; i < n; i++) {
    release(batch[i], prep[i]);
    batch[i]->status = rc[i];
  }
  // keep small workspaces for the next batch, free the large ones
  for (int i = 0; i < n; i++)
    if (pool[i]->bytes > KEEP_WS_BYTES) pool[i].reset(new Member());
  std::lock_guard<std::mutex> lk(mu);
  st.batches++;
  const double bms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  const double sms = std::chrono::duration<double, std::milli>(t2 - t1).count();
  st.build_ms += bms * n;
  st.solve_ms += sms * n;
}

void sx_server_s::worker(int slot) {
  (void)slot;
  cudaSetDevice(device);
  cudaStream_t stream = nullptr;
  cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
  sx_batch b = nullptr;
  sx_batch_create(&b);
  b->use_graphs = false;
  std::vector<std::unique_ptr<Member>> pool;
  for (;;) {
    std::vector<Req *> batch;
    {
      std::unique_lock<std::mutex> lk(mu);
      for (;;) {
        if (stopping && pending.empty()) break;
        // every admissible pending request, in arrival order, up to max_batch
        while (!pending.empty() && (int)batch.size() < cfg.max_batch) {
          Req *h = pending.front();
          size_t need = 0;
          if (!admissible(h, need)) evict_for(need, h->mesh.key);
          if (!(admissible(h, need) || (inflight == 0 && batch.empty()))) break;
          pending.pop_front();
          h->reserve = work_estimate(h->mesh, h->nz, cfg.precision);
          bytes_reserved += h->reserve;
          inflight++;
          st.queue_ms += std::chrono::duration<double, std::milli>(Clock::now() - h->t_submit).count();
          batch.push_back(h);
        }
        if (!batch.empty()) break;
        cv_work.wait(lk);
      }
    }
    if (batch.empty()) break;
    serve_batch(batch, pool, b, stream);
    {
      std::lock_guard<std::mutex> lk(mu);
      for (Req *r : batch) {
        r->latency_ms = std::chrono::duration<double, std::milli>(Clock::now() - r->t_submit).count();
        r->done = true;
        bytes_reserved -= r->reserve;
        inflight--;
        if (r->status == SX_OK || r->status == SX_WARN_STEP_LIMIT) {
          st.completed++;
          latencies.push_back(r->latency_ms);
        } else {
          st.failed++;
        }
        // drop the big copies now; the record stays for sx_server_wait
        r->f.clear();
        r->f.shrink_to_fit();
        r->bc.clear();
      }
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }
  pool.clear();
  sx_batch_destroy(b);
  cudaStreamDestroy(stream);
}

extern "C" int sx_server_create(const sx_server_config *cfg, sx_server *out) {
  if (!out) return SX_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<sx_server_s> S(new sx_server_s());
  if (cfg) S->cfg = *cfg;
  sx_server_config &c = S->cfg;
  if (c.precision != SX_FP64) c.precision = SX_MIXED_FP32;
  if (c.slots <= 0) c.slots = 4;
  if (c.slots > 64) return SX_ERR_ARG;
  if (c.tol_rel <= 0.0) c.tol_rel = 1e-12;
  if (c.max_refine <= 0) c.max_refine = 30;
  if (c.inner_iters <= 0) c.inner_iters = 12;
  if (c.max_batch <= 0) c.max_batch = 8;
  if (c.max_batch > 256) return SX_ERR_ARG;
  SX_CUDA(cudaGetDevice(&S->device));
  if (c.hbm_budget == 0) {
    size_t fr = 0, tot = 0;
    SX_CUDA(cudaMemGetInfo(&fr, &tot));
    c.hbm_budget = (unsigned long long)(0.8 * fr);
  }
  S->st.bytes_budget = c.hbm_budget;
  sx_server_s *p = S.get();
  for (int i = 0; i < c.slots; i++) S->workers.emplace_back([p, i]() { p->worker(i); });
  *out = S.release();
  return SX_OK;
}

extern "C" int sx_server_submit(sx_server s, const sx_request *q, unsigned long long *id) {
  if (!s || !q || !q->mesh || !q->f || !q->u || !q->lambda2 || !q->betak2 || q->num_modes <= 0 || q->nz <= 0)
    return SX_ERR_ARG;
  const sx_mesh_desc &d = *q->mesh;
  if (d.np < NP_MIN || d.np > NP_MAX || d.nel <= 0 || q->plane_stride < d.nel * d.np * d.np) return SX_ERR_ARG;
  if (q->nz > 1 && (q->nz % 2 || q->nz / 2 > q->num_modes)) return SX_ERR_ARG;
  std::unique_ptr<Req> r(new Req());
  MeshCopy &m = r->mesh;
  const size_t nn = (size_t)d.np * d.np, tb = (size_t)d.nel * 4 * (d.np - 1);
  m.np = d.np; m.nel = d.nel; m.nglobal = d.nglobal; m.nsolve = d.nsolve; m.nband = d.nband;
  m.nbound = d.nbound;
  m.x.assign(d.x, d.x + d.nel * nn);
  m.y.assign(d.y, d.y + d.nel * nn);
  m.btog.assign(d.btog, d.btog + tb);
  m.bmask.assign(d.bmask, d.bmask + tb);
  const int nb = std::max(d.nbound, 0);
  m.be.assign(nb + 1, 0); m.bs.assign(nb + 1, 0); m.bk.assign(nb + 1, 0);
  m.bK.assign(nb + 1, 0.0); m.bC.assign(nb + 1, 0.0);
  for (int b = 0; b < nb; b++) {
    m.be[b] = d.b_elmt[b]; m.bs[b] = d.b_side[b]; m.bk[b] = d.b_kind[b];
    if (d.b_K) m.bK[b] = d.b_K[b];
    if (d.b_C) m.bC[b] = d.b_C[b];
  }
  uint64_t h = 1469598103934665603ull;
  int hdr[6] = {m.np, m.nel, m.nglobal, m.nsolve, m.nband, m.nbound};
  h = fnv(h, hdr, sizeof(hdr));
  h = fnv(h, m.x.data(), m.x.size() * 8);
  h = fnv(h, m.y.data(), m.y.size() * 8);
  h = fnv(h, m.btog.data(), m.btog.size() * 4);
  h = fnv(h, m.bmask.data(), m.bmask.size() * 4);
  h = fnv(h, m.be.data(), m.be.size() * 4);
  h = fnv(h, m.bs.data(), m.bs.size() * 4);
  h = fnv(h, m.bk.data(), m.bk.size() * 4);
  h = fnv(h, m.bK.data(), m.bK.size() * 8);
  h = fnv(h, m.bC.data(), m.bC.size() * 8);
  m.key = h;
  {
    const int rk = mesh_kratio(&d, &m.kratio);
    if (rk != SX_OK) return rk;
  }
  r->base_mode = q->base_mode;
  r->num_modes = q->num_modes;
  r->nz = q->nz;
  r->stride = q->plane_stride;
  r->lam.assign(q->lambda2, q->lambda2 + q->num_modes);
  r->bk2.assign(q->betak2, q->betak2 + q->num_modes);
  r->f.assign(q->f, q->f + (size_t)q->nz * q->plane_stride);
  if (q->bc) r->bc.assign(q->bc, q->bc + (size_t)q->nz * std::max(d.nbound, 1) * d.np);
  r->u = q->u;
  r->t_submit = Clock::now();
  // a request that cannot fit even in an empty device is refused up front
  std::lock_guard<std::mutex> lk(s->mu);
  size_t alone = work_estimate(m, r->nz, s->cfg.precision) + mesh_estimate(m);
  for (int l = 0; l < r->num_modes; l++) alone += system_estimate(m, s->mode_kind(m, r->lam[l], r->bk2[l]));
  s->st.submitted++;
  if (alone > s->cfg.hbm_budget) {
    s->st.rejected++;
    set_error("request needs ~%zu bytes, budget %llu", alone, s->cfg.hbm_budget);
    return SX_ERR_CAPACITY;
  }
  r->id = s->next_id++;
  if (id) *id = r->id;
  s->pending.push_back(r.get());
  s->reqs[r->id] = std::move(r);
  s->cv_work.notify_one();
  return SX_OK;
}

extern "C" int sx_server_wait(sx_server s, unsigned long long id, double timeout_s, int *status,
                              double *latency_ms) {
  if (!s) return SX_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return SX_ERR_NOT_FOUND;
  Req *r = it->second.get();
  auto pred = [r]() { return r->done; };
  if (timeout_s < 0)
    s->cv_done.wait(lk, pred);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
    return SX_ERR_TIMEOUT;
  if (status) *status = r->status;
  if (latency_ms) *latency_ms = r->latency_ms;
  s->reqs.erase(it);
  return SX_OK;
}

extern "C" int sx_server_get_stats(sx_server s, sx_server_stats *out) {
  if (!s || !out) return SX_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  sx_server_stats st = s->st;
  st.bytes_cached = s->bytes_cached;
  std::vector<double> l = s->latencies;
  if (!l.empty()) {
    std::sort(l.begin(), l.end());
    auto q = [&](double f) { return l[std::min(l.size() - 1, (size_t)std::floor(f * (l.size() - 1) + 0.5))]; };
    st.p50_ms = q(0.50);
    st.p99_ms = q(0.99);
    double sum = 0.0;
    for (double v : l) sum += v;
    st.mean_ms = sum / l.size();
  }
  *out = st;
  return SX_OK;
}

extern "C" int sx_server_destroy(sx_server s) {
  if (!s) return SX_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (auto &t : s->workers) t.join();
  delete s;
  return SX_OK;
}
