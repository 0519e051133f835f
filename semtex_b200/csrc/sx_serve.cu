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
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <list>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "sx_modal.h"

using namespace sx;
namespace sx {
const char *last_error();
}
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
  size_t build_bytes = 0;  // estimate of the mesh and systems its build adds to the cache
  bool done = false;
  int status = SX_OK;
  double latency_ms = 0.0;
};

// Cache entries are inserted by the slot that builds them as soon as it
// starts, so that no two slots build the same entry; `ready` is set when the
// build is done (a mesh) or enqueued with its event recorded (a system), and
// `failed` when it went wrong.  A slot waits for other slots' entries only
// after marking its own ready, so waits cannot form a cycle.
struct MeshEntry {
  std::unique_ptr<sx_mesh_s> mesh;
  size_t bytes = 0;
  int refs = 0;
  uint64_t last_use = 0;
  bool ready = false, failed = false;
};

struct SysEntry {
  std::shared_ptr<System> sys;
  uint64_t mesh_key = 0;
  size_t bytes = 0;
  int refs = 0;
  uint64_t last_use = 0;
  bool ready = false, failed = false;
};

// Least time of one FP32 iteration of a serving batch (a launch from the host).
constexpr double SERVE_ITER_S = 12e-6;

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
  // band-solve workspace (rhs, condensed forcing, essential values): every
  // plane in the FP64 form, and any plane the mixed form routes to the band
  b += (size_t)nz * ((m.nsolve + NB) * 8 + (size_t)m.nel * next * 8 + (size_t)m.nglobal * 8);
  if (precision == SX_MIXED_FP32)  // node vectors, element vectors, FP64 element results, preconditioner
    b += PP * npts * (2 * 8 + 4) + PP * m.nel * nn * (6 * 4 + 8 + 2) + PP * m.nglobal * 8 + npts * (nz / 2 + 1) * 4;
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
  std::vector<std::thread> workers;
  std::vector<double> latencies;
  sx_server_stats st{};
  // SX_SERVER_TRACE set: one line per batch on stderr (its timeline)
  bool trace = false;
  Clock::time_point t_start = Clock::now();
  // Device memory of the cached systems and the workspaces: a pool grown to
  // the budget at creation, so that a build or a workspace sub-allocates in
  // stream order instead of paying a cudaMalloc (~0.2-1 ms each on B200)
  cudaMemPool_t mem_pool = nullptr;
  // Before a batch's builds: when the pool's free
  // reserve is below `need`, grow it by at least POOL_STEP in one allocation
  // freed at once on `stream`, so that the batch's allocations map nothing.
  static constexpr size_t POOL_STEP = size_t(4) << 30;
  void grow_pool(size_t need, cudaStream_t stream) {
    uint64_t reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(mem_pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess ||
        cudaMemPoolGetAttribute(mem_pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    if (reserved - used >= need) return;
    size_t step = std::max(need, POOL_STEP);
    if (reserved + step > cfg.hbm_budget) step = cfg.hbm_budget > reserved ? cfg.hbm_budget - reserved : 0;
    void *p = nullptr;
    if (step > 0 && cudaMallocFromPoolAsync(&p, step, mem_pool, stream) == cudaSuccess) cudaFreeAsync(p, stream);
    cudaGetLastError();  // best effort: the pool still grows on demand
  }
  // After a batch: requests of many sizes leave the pool fragmented, and
  // it grows by new mappings where a free run is too short; once its
  // reserved memory passes the budget, hand the unused part back (the
  // allocations in use stay), so that the device never fills up with free
  // pool memory that a plain cudaMalloc (mesh tables) cannot use.
  void trim_pool(cudaStream_t stream) {
    uint64_t reserved = 0;
    if (cudaMemPoolGetAttribute(mem_pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    if (reserved <= cfg.hbm_budget) return;
    cudaStreamSynchronize(stream);  // this slot's frees are complete
    cudaMemPoolTrimTo(mem_pool, (size_t)(0.75 * (double)cfg.hbm_budget));
    cudaGetLastError();
  }
  ~sx_server_s() {
    systems.clear();
    meshes.clear();
    if (mem_pool) {
      cudaDeviceSynchronize();  // the frees above are stream-ordered
      cudaMemPoolDestroy(mem_pool);
    }
  }

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
    // The serving loop's FP32 iterations are launched one by one from the
    // host (a batch's member set changes from batch to batch, so nothing is
    // captured) with the host checking every round: at least SERVE_ITER_S
    // an iteration, and the iteration model is charged twice over (measured
    // on serving-sized meshes, lambda2 = 10 + k^2: 32 x 32, N = 7, 32 modes:
    // Jacobi-CG 124 ms against a band build of 93 ms and a 3 ms solve;
    // 64 x 64, N = 10, 64 modes: 6.5 s against 3.3 s and 45 ms).
    return band_cheaper(m.np, m.nel, m.nglobal, m.nsolve, m.nband, m.kratio, lam + bk2, cfg.inner_iters,
                        cfg.tol_rel, cfg.max_refine, 1.0, SERVE_ITER_S, 2.0)
               ? SX_DIRECT
               : SX_JACPCG;
  }
  bool admissible(Req *r, size_t &need);
  void evict_for(size_t need, uint64_t keep_mesh);
  // After a batch (caller holds mu): the cache keeps at most a quarter of the
  // budget of entries no request is using.  A stream whose requests rarely
  // share a system (each carries its own lambda2) gains nothing from a full
  // cache, and a pool that holds the whole budget in systems of every size
  // fragments until its reserved memory fills the device.
  void trim_cache() {
    const size_t budget = (size_t)cfg.hbm_budget, cap = budget / 4;
    if (bytes_cached > cap) evict_for(budget - cap - std::min(bytes_reserved, budget - cap), 0);
  }
  void worker(int slot);
  using SysKey = std::tuple<uint64_t, uint64_t, uint64_t, int>;
  // One request's mesh and systems.
  struct Prep {
    double mesh_ms = 0.0, direct_ms = 0.0, jacobi_ms = 0.0;  // host time of the builds (trace)
    sx_mesh_s *mesh = nullptr;
    std::vector<std::shared_ptr<System>> sys;
    std::vector<SysKey> keys;     // every entry this request holds a reference on
    std::vector<SysKey> built;    // entries this slot builds
    std::vector<SysKey> foreign;  // entries another slot was still building
    bool mesh_ref = false;
  };
  // Look up one request's mesh and systems, and enqueue on `stream`, without
  // waiting, the builds of those the cache lacks; new band factors are
  // appended to to_factor.
  int prepare(Req *r, Prep &p, std::vector<System *> &to_factor, cudaStream_t stream);
  std::condition_variable cv_ready;  // a cache entry became ready
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
  for (int l = 0; l < r->num_modes; l++) r->kinds[l] = mode_kind(r->mesh, r->lam[l], r->bk2[l]);
  // One request's new band factors may take at most a quarter of the budget
  // (the largest request of the serving stream, 64 x 64 elements at N = 10
  // with 64 modes, would need ~113 GB): past that, the modes with the
  // largest Helmholtz constant, whose FP32 iterations converge fastest, go to
  // the iterations instead (mixed precision only; the FP64 server refuses
  // what cannot fit).
  auto key_of = [&](int l, int kind) {
    uint64_t a, b;
    std::memcpy(&a, &r->lam[l], 8);
    std::memcpy(&b, &r->bk2[l], 8);
    return std::make_tuple(r->mesh.key, a, b, kind);
  };
  if (cfg.precision == SX_MIXED_FP32) {
    const size_t cap = cfg.hbm_budget / 4, per = system_estimate(r->mesh, SX_DIRECT);
    size_t band = 0;
    std::vector<int> order;
    for (int l = 0; l < r->num_modes; l++)
      if (r->kinds[l] == SX_DIRECT && !systems.count(key_of(l, SX_DIRECT))) {
        band += per;
        order.push_back(l);
      }
    std::sort(order.begin(), order.end(),
              [&](int a, int b) { return r->lam[a] + r->bk2[a] > r->lam[b] + r->bk2[b]; });
    for (size_t i = 0; i < order.size() && band > cap; i++) {
      r->kinds[order[i]] = SX_JACPCG;
      band -= per;
    }
  }
  for (int l = 0; l < r->num_modes; l++)
    if (!systems.count(key_of(l, r->kinds[l]))) need += system_estimate(r->mesh, r->kinds[l]);
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
  auto since = [](Clock::time_point a) { return std::chrono::duration<double, std::milli>(Clock::now() - a).count(); };
  bool build_mesh = false;
  {
    std::unique_lock<std::mutex> lk(mu);
    auto it = meshes.find(r->mesh.key);
    if (it != meshes.end()) {
      it->second.refs++;
      it->second.last_use = ++tick;
      pp.mesh_ref = true;
      st.mesh_hits++;
      // a mesh another slot is creating: its creation waits for nothing
      MeshEntry &e = it->second;
      cv_ready.wait(lk, [&]() { return e.ready; });
      if (e.failed) return SX_ERR_CUDA;
      pp.mesh = e.mesh.get();
    } else {
      MeshEntry &e = meshes[r->mesh.key];
      e.bytes = mesh_estimate(r->mesh);
      e.refs = 1;
      e.last_use = ++tick;
      bytes_cached += e.bytes;
      pp.mesh_ref = true;
      st.mesh_misses++;
      build_mesh = true;
    }
  }
  if (build_mesh) {
    const auto tm = Clock::now();
    const sx_mesh_desc d = r->mesh.desc();
    sx_mesh m = nullptr;
    const int rc = sx_mesh_create(&d, &m);
    {
      std::lock_guard<std::mutex> lk(mu);
      MeshEntry &e = meshes[r->mesh.key];
      e.mesh.reset(m);
      e.ready = true;
      e.failed = rc != SX_OK;
    }
    cv_ready.notify_all();
    SX_TRY(rc);
    pp.mesh = m;
    pp.mesh_ms += since(tm);
  }
  pp.sys.resize(r->num_modes);
  for (int l = 0; l < r->num_modes; l++) {
    const int kind = r->kinds[l];
    uint64_t a, b;
    std::memcpy(&a, &r->lam[l], 8);
    std::memcpy(&b, &r->bk2[l], 8);
    const SysKey key = std::make_tuple(r->mesh.key, a, b, kind);
    std::shared_ptr<System> S;
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = systems.find(key);
      if (it != systems.end()) {
        pp.sys[l] = it->second.sys;
        it->second.refs++;
        it->second.last_use = ++tick;
        pp.keys.push_back(key);
        st.system_hits++;
        if (!it->second.ready && std::find(pp.built.begin(), pp.built.end(), key) == pp.built.end())
          pp.foreign.push_back(key);
        continue;
      }
      S = std::make_shared<System>();
      S->pool = mem_pool;
      S->mesh = pp.mesh;
      S->lambda2 = r->lam[l];
      S->betak2 = r->bk2[l];
      S->method = kind;
      SysEntry &e = systems[key];
      e.sys = S;
      e.mesh_key = r->mesh.key;
      e.bytes = system_estimate(r->mesh, kind);
      e.refs = 1;
      e.last_use = ++tick;
      bytes_cached += e.bytes;
      pp.keys.push_back(key);
      pp.built.push_back(key);
      st.system_misses++;
    }
    pp.sys[l] = S;
    const auto tb = Clock::now();
    if (kind == SX_DIRECT) {
      SX_TRY(system_build_direct(*S, stream, false));
      if (S->nsolve > 0) to_factor.push_back(S.get());
      SX_TRY(system_build_jacobi_diag(*S, stream, false));
      pp.direct_ms += since(tb);
    } else {
      SX_TRY(system_build_jacobi(*S, stream, false));
      pp.jacobi_ms += since(tb);
    }
  }
  return SX_OK;
}

// Drop the request's references (caller has synchronised the slot's
// stream, so no work of this batch is in flight); an entry whose build
// failed leaves the cache with its last reference, so that a later request
// builds it again.
void sx_server_s::release(const Req *r, const Prep &pp) {
  std::lock_guard<std::mutex> lk(mu);
  for (auto &k : pp.keys) {
    auto si = systems.find(k);
    if (si == systems.end()) continue;
    if (--si->second.refs == 0 && si->second.failed) {
      bytes_cached -= si->second.bytes;
      systems.erase(si);
    }
  }
  if (pp.mesh_ref) {
    auto mi = meshes.find(r->mesh.key);
    if (mi != meshes.end() && --mi->second.refs == 0 && mi->second.failed) {
      bool used = false;
      for (auto &s : systems)
        if (s.second.mesh_key == mi->first) used = true;
      if (!used) {
        bytes_cached -= mi->second.bytes;
        meshes.erase(mi);
      }
    }
  }
}

// Memory estimate (workspace plus new cache entries) up to which admitted
// requests are gathered into one batch.
constexpr size_t BATCH_BYTES = size_t(1) << 30;

// Workspaces above this size are freed after their batch instead of kept
// for the next one (a pool slot otherwise holds the largest request it saw).
constexpr size_t KEEP_WS_BYTES = size_t(256) << 20;

void sx_server_s::serve_batch(std::vector<Req *> &batch, std::vector<std::unique_ptr<Member>> &pool, sx_batch b,
                              cudaStream_t stream) {
  const int n = (int)batch.size();
  const auto t0 = Clock::now();
  std::vector<Prep> prep(n);
  std::vector<int> rc(n, SX_OK);
  Clock::time_point tl, tf;
  size_t nfactor = 0;
  {
    // look up the meshes and systems, enqueue the builds of the missing ones
    // and one factorisation of the batch's new band systems, all on this
    // slot's stream without waiting (other slots build theirs meanwhile); an
    // event recorded after them marks the new systems ready for the other
    // slots' streams
    tl = Clock::now();
    size_t need = 0;
    for (int i = 0; i < n; i++) need += batch[i]->reserve + batch[i]->build_bytes;
    grow_pool(need, stream);
    std::vector<System *> to_factor;
    for (int i = 0; i < n; i++) rc[i] = prepare(batch[i], prep[i], to_factor, stream);
    tf = Clock::now();
    nfactor = to_factor.size();
    int fr = factor_batch(to_factor, stream, false);
    auto ev = std::make_shared<ReadyEvent>();
    if (fr == SX_OK && (cudaEventCreateWithFlags(&ev->ev, cudaEventDisableTiming) != cudaSuccess ||
                        cudaEventRecord(ev->ev, stream) != cudaSuccess)) {
      set_error("serving: could not record a build event");
      fr = SX_ERR_CUDA;
    }
    {
      // this slot's new entries are ready (or failed) for everyone
      std::lock_guard<std::mutex> lk(mu);
      for (int i = 0; i < n; i++) {
        if (fr != SX_OK && rc[i] == SX_OK) rc[i] = fr;
        for (auto &k : prep[i].built) {
          auto it = systems.find(k);
          if (it == systems.end()) continue;
          it->second.sys->ready = ev;
          it->second.ready = true;
          it->second.failed = rc[i] != SX_OK;
        }
      }
    }
    cv_ready.notify_all();
    // then the entries other slots were building
    std::unique_lock<std::mutex> lk(mu);
    for (int i = 0; i < n; i++)
      for (auto &k : prep[i].foreign) {
        auto it = systems.find(k);
        if (it == systems.end()) continue;
        SysEntry &e = it->second;
        cv_ready.wait(lk, [&]() { return e.ready; });
        if (e.failed && rc[i] == SX_OK) rc[i] = SX_ERR_CUDA;
      }
  }
  // systems another slot built: wait (on the device) for their builds
  for (int i = 0; i < n; i++)
    for (auto &S : prep[i].sys)
      if (S && S->ready && S->ready->ev && cudaStreamWaitEvent(stream, S->ready->ev, 0) != cudaSuccess)
        rc[i] = SX_ERR_CUDA;
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
      m.ws->pool = mem_pool;
      m.ws->mixed.pool = mem_pool;
    }
    sx_modal_s &ws = *m.ws;
    ws.rebind(prep[i].mesh, r->base_mode, r->num_modes, cfg.precision == SX_FP64 ? SX_DIRECT : SX_MIXED,
              prep[i].sys);
    ws.n_inner = cfg.inner_iters;
    const size_t len = (size_t)r->nz * r->stride;
    int e = SX_OK;
    if (m.du.n < len) e = m.du.alloc_in(len, mem_pool, stream);
    if (e == SX_OK && m.df.n < len) e = m.df.alloc_in(len, mem_pool, stream);
    if (e == SX_OK && !r->bc.empty() && m.dbc.n < r->bc.size())
      e = m.dbc.alloc_in(r->bc.size(), mem_pool, stream);
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
    // the systems' build statuses (interior blocks, band factors)
    for (size_t k = 0; k < idx.size(); k++)
      for (auto &S : prep[idx[k]].sys) {
        const int c = S ? system_check_status(*S) : SX_OK;
        if (c != SX_OK) rc[idx[k]] = c;
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
  // builds enqueued for requests that failed before the solve may still run
  if (cudaStreamSynchronize(stream) != cudaSuccess)
    for (int i = 0; i < n; i++) rc[i] = rc[i] == SX_OK ? SX_ERR_CUDA : rc[i];
  const auto t2 = Clock::now();
  for (int i = 0; i < n; i++) {
    release(batch[i], prep[i]);
    batch[i]->status = rc[i];
  }
  // keep small workspaces for the next batch, free the large ones; a kept
  // workspace lets go of the request's systems (it would otherwise keep
  // them alive after the cache has evicted them and stopped counting them)
  for (int i = 0; i < n; i++) {
    if (pool[i]->bytes > KEEP_WS_BYTES)
      pool[i].reset(new Member());
    else if (pool[i]->ws)
      pool[i]->ws->rebind(nullptr, 0, 0, pool[i]->ws->method, {});
  }
  trim_pool(stream);
  std::lock_guard<std::mutex> lk(mu);
  trim_cache();
  st.batches++;
  auto ms = [](Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
  };
  st.build_ms += ms(t0, t1) * n;
  st.solve_ms += ms(t1, t2) * n;
  if (trace) {
    double mm = 0.0, dm = 0.0, jm = 0.0;
    for (auto &p : prep) {
      mm += p.mesh_ms;
      dm += p.direct_ms;
      jm += p.jacobi_ms;
    }
    size_t fr = 0, tot = 0;
    uint64_t pres = 0, pused = 0;
    cudaMemGetInfo(&fr, &tot);
    cudaMemPoolGetAttribute(mem_pool, cudaMemPoolAttrReservedMemCurrent, &pres);
    cudaMemPoolGetAttribute(mem_pool, cudaMemPoolAttrUsedMemCurrent, &pused);
    cudaGetLastError();
    std::fprintf(stderr,
                 "sx_server batch %llu: %d requests, t=%.1f ms, build %.1f (meshes %.1f, band systems %.1f, "
                 "Jacobi %.1f), factor and waits %.1f (%zu systems factored), solve %.1f | device free %.1f GB, "
                 "pool %.1f / %.1f GB, cached %.1f GB (%zu meshes, %zu systems), reserved %.1f GB\n",
                 (unsigned long long)st.batches, n, ms(t_start, t0), ms(tl, tf), mm, dm, jm, ms(tf, t1), nfactor,
                 ms(t1, t2), fr / 1e9, pused / 1e9, pres / 1e9, bytes_cached / 1e9, meshes.size(), systems.size(),
                 bytes_reserved / 1e9);
    for (int i = 0; i < n; i++)
      if (rc[i] != SX_OK && rc[i] != SX_WARN_STEP_LIMIT)
        std::fprintf(stderr, "sx_server   request %llu failed: status %d (%s)\n", (unsigned long long)batch[i]->id,
                     rc[i], sx::last_error());
  }
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
        // admissible pending requests in arrival order, up to max_batch, and
        // while the batch's memory estimate stays under BATCH_BYTES: small
        // requests share a batch, a large one (whose builds and iterations
        // would hold up the small ones) is served by itself
        size_t batch_bytes = 0;
        while (!pending.empty() && (int)batch.size() < cfg.max_batch) {
          Req *h = pending.front();
          size_t need = 0;
          if (!admissible(h, need)) evict_for(need, h->mesh.key);
          if (!(admissible(h, need) || (inflight == 0 && batch.empty()))) break;
          if (!batch.empty() && batch_bytes + need > BATCH_BYTES) break;
          batch_bytes += need;
          pending.pop_front();
          h->reserve = work_estimate(h->mesh, h->nz, cfg.precision);
          h->build_bytes = need > h->reserve ? need - h->reserve : 0;
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
  if (c.slots <= 0) c.slots = 8;
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
    c.hbm_budget = (unsigned long long)(0.7 * fr);
  }
  S->st.bytes_budget = c.hbm_budget;
  {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = S->device;
    SX_CUDA(cudaMemPoolCreate(&S->mem_pool, &props));
    // hold on to freed memory up to a quarter of the budget (a
    // sub-allocation from the pool costs microseconds, a fresh mapping up to
    // a millisecond); above it the pool hands unused memory back at
    // synchronisation points, for the allocations made outside it
    uint64_t keep = c.hbm_budget / 4;
    SX_CUDA(cudaMemPoolSetAttribute(S->mem_pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  S->trace = std::getenv("SX_SERVER_TRACE") != nullptr;
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
