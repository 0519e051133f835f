// sx_internal.h -- shared declarations of the semtex_b200 library (not part
// of the public C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/semtex_b200.h"

namespace sx {

// Reference tolerances (veclib/utility.h:35,39).
constexpr double EPSSP = 6.0e-7;
constexpr double EPSDP = 6.0e-14;

// Band tiles: the condensed matrix is held as nb x nb tiles; tile (k, j)
// holds U(rows of block k-j, cols of block k).  Rows are padded to
// LDT = NB + 1 doubles so that both row- and column-wise smem traversals
// are free of bank conflicts.
constexpr int NB = 64;
constexpr int LDT = NB + 1;
constexpr int TSZ = NB * LDT;  // doubles per tile (33280 B, 16-B multiple)

constexpr int NP_MIN = 3;
constexpr int NP_MAX = 12;

struct Status {
  int code = SX_OK;
  std::string msg;
};

// Thread-local last error message, for sx_status_string callers.
void set_error(const char *fmt, ...);

// GLL points, weights and derivative matrix (row-major D[i][j] = h_j'(z_i)).
void gll_tables(int np, std::vector<double> &z, std::vector<double> &w, std::vector<double> &D);

#define SX_CUDA(call)                                                                  \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      ::sx::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
      return (e_ == cudaErrorMemoryAllocation) ? SX_ERR_NOMEM : SX_ERR_CUDA;          \
    }                                                                                  \
  } while (0)

#define SX_TRY(call)            \
  do {                          \
    int s_ = (call);            \
    if (s_ != SX_OK) return s_; \
  } while (0)

// Device buffer with RAII release.
// alloc()/upload() use cudaMalloc (long-lived data); alloc_on()/upload_on()
// use the stream-ordered allocator on a stream, so releasing a temporary
// never synchronises the device (cudaFree would).
template <typename T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  bool ordered = false;
  cudaStream_t os = nullptr;
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) {
      if (ordered)
        cudaFreeAsync(p, os);
      else
        cudaFree(p);
    }
    p = nullptr;
    n = 0;
    ordered = false;
  }
  int alloc_on(size_t count, cudaStream_t s) {
    release();
    if (count == 0) count = 1;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&p), count * sizeof(T), s);
    if (e != cudaSuccess) {
      p = nullptr;
      set_error("cudaMallocAsync(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
      return SX_ERR_NOMEM;
    }
    n = count;
    ordered = true;
    os = s;
    return SX_OK;
  }
  int upload_on(const T *h, size_t count, cudaStream_t s) {
    SX_TRY(alloc_on(count, s));
    SX_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    return SX_OK;
  }
  int alloc(size_t count) {
    release();
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      set_error("cudaMalloc(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
      return SX_ERR_NOMEM;
    }
    n = count;
    return SX_OK;
  }
  // From `pool` on stream s (stream-ordered, no device-wide synchronisation);
  // plain alloc when pool is null.  Freed on s when free_on_s (a temporary
  // whose last use is on s), else on the legacy stream (valid after s is
  // gone: the owner frees it only when no enqueued work uses it).
  int alloc_in(size_t count, cudaMemPool_t pool, cudaStream_t s, bool free_on_s = false) {
    if (!pool) return free_on_s ? alloc_on(count, s) : alloc(count);
    release();
    if (count == 0) count = 1;
    cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&p), count * sizeof(T), pool, s);
    if (e != cudaSuccess) {
      p = nullptr;
      set_error("cudaMallocFromPoolAsync(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
      return SX_ERR_NOMEM;
    }
    n = count;
    ordered = true;
    os = free_on_s ? s : nullptr;
    return SX_OK;
  }
  // From `pool` (alloc_in), copied on stream s and complete on return (the
  // wait is for s alone, not the device)
  int upload_in(const T *h, size_t count, cudaMemPool_t pool, cudaStream_t s) {
    SX_TRY(alloc_in(count, pool, s));
    SX_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    SX_CUDA(cudaStreamSynchronize(s));
    return SX_OK;
  }
  int upload(const T *h, size_t count) {
    SX_TRY(alloc(count));
    SX_CUDA(cudaMemcpy(p, h, count * sizeof(T), cudaMemcpyHostToDevice));
    return SX_OK;
  }
  int zero(cudaStream_t s = 0) {
    SX_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
    return SX_OK;
  }
};

// Device-side view of a mesh, passed by value to kernels.
struct MeshView {
  int np, npnp, next, nint, nel;
  int nglobal, nsolve_ns, nband;
  const double *D;       // np*np row-major, D[i][j] = h_j'(z_i)
  const int *emap;       // npnp
  const double *Q1, *Q2, *Q3, *Q4, *Q8;  // nel*npnp (Q3 zero when absent)
  const float *Q1f, *Q2f, *Q3f, *Q4f;    // FP32 copies (mixed precision)
  const float *Df;                       // FP32 copy of D
  const unsigned char *hasQ3;            // nel
  const int *btog, *bmask, *emask;       // nel*next, nel*next, nel
  const int *g2e_ptr, *g2e_idx;          // CSR: global node -> (e*next+i), element order
  const int *g2e_last;                   // nglobal: last (e*next+i) writing node (local2global)
  const int4 *g2e4;                      // nglobal: first 4 CSR entries, -1 padded, .w = -2 if more
  const unsigned long long *owner;       // nel: bit a set when element e is node btog[e][a]'s last writer
  const int4 *e2w4;                      // nel*next: gather list of node btog[e][a], in CSR order, as
                                         // (element << 8 | tensor node) of its first four holders,
                                         // -1 padded, .w = -2 when it has more (walk the CSR)
  const float4 *Gf;                      // nel*npnp: (Q1, Q2, Q3, Q4) in FP32, tensor order
  const int *pmap;                       // npnp: edge-map slot of tensor node t (inverse of emap)
  int nbound;
  const int *b_elmt, *b_side, *b_kind;
  const double *b_K, *b_C, *b_area;      // b_area: nbound*np
  const int *nat_ptr, *nat_idx;          // CSR: global node -> (b*np+i) natural/mixed terms
  int mixed;                             // any mixed boundary
};

struct sx_mesh_impl;
struct System;

}  // namespace sx

struct sx_mesh_s {
  int device = 0;
  int np = 0, npnp = 0, next = 0, nint = 0, nel = 0;
  int nglobal = 0, nsolve = 0, nband = 0, nbound = 0;
  bool mixed = false;
  std::vector<double> z, w, D;
  std::vector<int> emap, pmap;
  std::vector<double> Q1, Q2, Q3, Q4, Q8;  // host copies
  // inverse mapping partials dr/dx, dr/dy, ds/dx, ds/dy (zero where the
  // reference's null-mapping drops them) and the inverse of the assembled
  // boundary mass (BoundarySys imass)
  std::vector<double> drdx, drdy, dsdx, dsdy, imass;
  std::vector<unsigned char> hasQ3;
  std::vector<int> btog, bmask, emask;
  std::vector<int> b_elmt, b_side, b_kind;
  std::vector<double> b_K, b_C, b_area;
  std::vector<int> colour_ptr, colour_elmt;  // element colouring (no shared nodes)
  // device
  sx::DBuf<double> dD, dQ1, dQ2, dQ3, dQ4, dQ8, dK, dC, darea;
  sx::DBuf<double> ddrdx, ddrdy, ddsdx, ddsdy, dimass;
  sx::DBuf<float> dQ1f, dQ2f, dQ3f, dQ4f, dDf;
  sx::DBuf<unsigned char> dhasQ3;
  sx::DBuf<int> dpmap;
  sx::DBuf<int> demap, dbtog, dbmask, demask, dg2e_ptr, dg2e_idx, dg2e_last, dbe, dbs, dbk;
  sx::DBuf<int> dnat_ptr, dnat_idx, dcolour_elmt;
  sx::DBuf<int4> dg2e4, de2w4;
  sx::DBuf<float4> dGf;
  // max over nodes of the assembled stiffness diagonal over the assembled
  // mass diagonal: the Jacobi-scaled operator's condition number is about
  // 1 + kratio / hCon
  double kratio = 0.0;
  // Envelope of the band factor in tiles of NB: for the env_nblk block
  // columns of nsolve, env[k] = off-diagonal tiles of block column k that
  // can be non-zero (above the diagonal), env[env_nblk + k] = those of block
  // row k (right of it).  Every other tile of the band is an exact zero.
  int env_nblk = 0;
  std::vector<int> env;
  sx::DBuf<int> denv;
  sx::DBuf<unsigned long long> downer;
  sx::MeshView view() const;
};

namespace sx {

// A CUDA event shared by the systems one build enqueued: recorded after
// their last kernel, waited on by streams that use them.
struct ReadyEvent {
  cudaEvent_t ev = nullptr;
  ReadyEvent() = default;
  ReadyEvent(const ReadyEvent &) = delete;
  ReadyEvent &operator=(const ReadyEvent &) = delete;
  ~ReadyEvent() {
    if (ev) cudaEventDestroy(ev);
  }
};

// One MatrixSys: a (lambda2, betak2, method) system on a mesh.
struct System {
  sx_mesh_s *mesh = nullptr;
  double lambda2 = 0.0, betak2 = 0.0;
  int method = SX_DIRECT;
  bool singular = false;
  int nsolve = 0;
  int nblk = 0, J = 0;     // band tiles: nblk block columns, J off-diagonal tiles
  DBuf<double> tiles;      // nblk*(J+1)*TSZ
  DBuf<double> dinv;       // nblk*TSZ: inverse of the diagonal U tiles
  DBuf<double> hbi;        // nel*next*nint  (hbi hii^-1, row-major next x nint)
  DBuf<double> hii;        // nel*nint*nint  (hii^-1, column-major)
  DBuf<float> hbif, hiif;  // FP32 copies for the mixed form
  DBuf<double> pc;         // npts: inverse Jacobi diagonal (JACPCG)
  DBuf<float> pcf;         // FP32 copy
  DBuf<int> status;        // device status bits (1 << SX_ERR_*)
  // set when the build was enqueued without waiting for it: streams other
  // than the builder's wait on it before using the system
  std::shared_ptr<ReadyEvent> ready;
  cudaMemPool_t pool = nullptr;  // when set, the builders allocate from it
  size_t bytes() const;
};

// Builders.  sync = false enqueues on st and returns without waiting: the
// caller synchronises st (or records an event) and then calls
// system_check_status.
int system_build_direct(System &S, cudaStream_t st, bool sync = true);
int system_build_jacobi(System &S, cudaStream_t st, bool sync = true);
int system_build_jacobi_diag(System &S, cudaStream_t st, bool sync = true);
int system_check_status(System &S);
int system_band_export(const System &S, double *ab);  // LAPACK band, host

// sx_mesh_s::kratio of a mesh description, from host geometry alone.
int mesh_kratio(const sx_mesh_desc *d, double *out);

// FP32 CG iterations one refinement round needs to cut its residual by
// 1e-6, about what FP32 arithmetic allows: Jacobi-CG takes about
// 5.3 sqrt(1 + kratio / hcon) iterations per 1e-7 (measured with the oracle
// over lambda2 = 1..1e6, N = 4..10, square and 1:4 elements: within +-40 %).
// Above CG_ROUND_CAP (or for hcon <= 0) the FP32 iterations are not used.
constexpr int CG_ROUND_CAP = 400;
int cg_round_iters(double kratio, double hcon);

// Whether the FP64 band Cholesky is the better route for one mode (two
// planes) of the mixed-precision form with Helmholtz constant hcon, solved
// to tol_rel with at least n_inner FP32 iterations per refinement round and
// at most max_refine rounds.  Predicted streaming times on B200 (the
// per-launch latencies are shared by all modes of a batched launch, so a
// mode is charged only for its bytes):
//   CG:     rounds of max(n_inner, cg_round_iters) iterations, one round per
//           1e-6 of tol_rel; each iteration streams 4 (8 npts + 2 nel np^2)
//           bytes per plane at 2.1 TB/s
//   band:   the factor twice plus hbi/hii at 1.9 TB/s
//   factor: nsolve nband^2 flops at 3.9 TFLOP/s (config-2 set-up,
//           measured), divided by `reuse`, the solves expected per factored
//           system (0: already factored, no cost).
// The two streaming rates are calibration constants: k_cg's and
// k_band_sweep's rates when the rule was set up.  Both kernels are faster
// now (about 2.7 and 2.8 TB/s); with those rates the rule sends more modes
// of a serving request to the band, and a request's factorisation, whose
// block-column steps are latency-bound, costs more than the flop estimate
// above -- the serving stream ran slower (makespan 7.2-7.7 s against
// 5.3-7.8 s in an A/B on one box), so the calibrated pair stays.
// A mode whose rounds would exceed CG_ROUND_CAP iterations, or whose CG would
// need more than max_refine rounds, goes to the band.  iter_floor_s is the
// least time an FP32 iteration takes whatever its bytes (a launch and, when
// the iterations are not replayed from a captured graph, the host's issue
// of it), iter_factor a margin on the iteration model.
bool band_cheaper(int np, int nel, int nglobal, int nsolve, int nband, double kratio, double hcon, int n_inner,
                  double tol_rel, int max_refine, double reuse, double iter_floor_s = 0.0, double iter_factor = 1.0);

// Solve workspace for up to `planes` planes of one system.
struct Work {
  int planes = 0;
  DBuf<double> Fb;      // planes*nel*next condensed element boundary forcing
  DBuf<double> rhs;     // planes*npad
  DBuf<double> gess;    // planes*nglobal essential values
  DBuf<int> status;     // device status word
  int reserve(const sx_mesh_s &M, int planes, int npad);
};

// Direct solve of P planes that share system S (P <= 2 in the plain form).
// u, f: plane pointers (device), bc: plane bc lines (device) or nullptr.
int direct_solve_planes(const System &S, Work &W, double *const *u, double *const *f,
                        const double *const *bc, int P, cudaStream_t st);

}  // namespace sx
