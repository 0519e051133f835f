// sx_band.cu -- banded triangular solves U^T y = b, U x = y (LAPACK
// dpbtrs "U" as called at src/field.cpp:609) on the tiled band factor.
//
// Both sweeps are left-looking over block columns of NB rows:
//   forward  y_k = D_k^T (b_k - sum_{j>=1} T(k,j)^T   y_{k-j})
//   backward x_k = D_k   (y_k - sum_{j>=1} T(k+j,j)   x_{k+j})
// with T(k,j) = U(rows of block k-j, cols of block k) and D_k = U_kk^-1.
//
// One thread-block cluster of C CTAs works on one system (all P right-hand
// sides of the job at once).  The leader CTA (rank 0) owns the critical
// path: the j = 1 tile (needs the block just solved) and D_k; ranks 1..C-1
// own the older tiles j >= 2 round-robin, so they run ahead while the
// leader finishes the previous block.  Tiles stream into each CTA through a
// ring of 1-D TMA bulk copies (cp.async.bulk + mbarrier complete_tx).
// Partial sums go to the leader over distributed shared memory; each solved
// block goes to the RHS array in global memory (where it stays in L2), and
// the leader's release at cluster scope on every rank's mbarrier for that
// block lets the ranks fetch it from there (cp.async through L2, one block
// per tile, issued under the previous tile's work).  Partials are combined
// in rank order, so the result does not depend on timing.
//
// Every wait is bounded (clock64); on timeout the kernel records
// SX_ERR_TIMEOUT in the status word, drains its own bulk copies (bounded),
// meets the other CTAs at a final cluster barrier and returns.
#include <algorithm>

#include "sx_kernels.cuh"
#include "sx_ptx.cuh"
#include "sx_solve.cuh"

namespace sx {

constexpr long long WAIT_LIMIT = SWEEP_WAIT_DEFAULT;  // ~2 s at 1.9 GHz


// Cycles a wait of the sweep loop may take before the kernel gives up
// (SX_ERR_TIMEOUT); per device, set by sx_set_wait_limit.  The drain of a
// CTA's own bulk copies on the way out always uses WAIT_LIMIT: those copies
// read valid memory and land within microseconds, and a CTA must not leave
// with copies into its shared memory still in flight.
__device__ long long g_sweep_wait = WAIT_LIMIT;

int set_sweep_wait_limit(long long cycles) {
  SX_CUDA(cudaMemcpyToSymbol(g_sweep_wait, &cycles, sizeof(cycles)));
  return SX_OK;
}

// Division by a small runtime divisor d (1 <= d <= 2^16) of n < 2^24 by one
// 64-bit multiply: floor(n / d) = (n ceil(2^40 / d)) >> 40 exactly in that
// range (the rounding error of the reciprocal stays below 2^-16 <= 1 / d).
struct FastDiv {
  unsigned long long m = 1ull << 40;
  unsigned d = 1;
  __host__ __device__ FastDiv() {}
  __host__ __device__ explicit FastDiv(unsigned dv) : m(((1ull << 40) + dv - 1) / dv), d(dv) {}
  __device__ __forceinline__ int div(int n) const { return (int)(((unsigned long long)(unsigned)n * m) >> 40); }
  __device__ __forceinline__ int mod(int n) const { return n - div(n) * (int)d; }
};

struct SweepGeom {
  int nblk, J, C, rank;
  // Leader share: Q = 0, the leader (rank 0) owns only the j = 1 tile and
  // D_k, and ranks 1..C-1 the tiles j >= 2 round-robin.  Q = K >= 2: the
  // positions p = j - 2 of the tiles j >= 2 run in cycles of K whose last
  // position is the leader's; the other positions go round-robin to ranks
  // 1..C-1.  The leader works through its tiles of step t + 1 during step t,
  // between its j = 1 tile and the wait for the ranks' partial sums, so they
  // stay off the block-column chain; they are listed under step t, after
  // the j = 1 tile and before D_k.
  int Q;
  FastDiv dC1, dQ, dQ1;  // divisions by C - 1, Q and Q - 1 (1 when unused)
  // Envelope of the factor (null: the whole band): jf[k] tiles above the
  // diagonal are non-zero in block column k, jb[k] right of it in block row
  // k; every tile beyond them is an exact zero and is skipped.
  const int *jf, *jb;
  // off-diagonal tiles of step t (t < nblk: forward block t, else backward
  // block 2 nblk - 1 - t)
  __device__ __forceinline__ int jmax(int t) const {
    if (t >= 2 * nblk) return 0;
    if (t < nblk) {
      const int b = min(J, t);
      return jf ? max(0, min(b, __ldg(jf + t))) : b;
    }
    const int k = 2 * nblk - 1 - t, b = min(J, nblk - 1 - k);
    return jb ? max(0, min(b, __ldg(jb + k))) : b;
  }
  // what a step's tile list depends on: its own tile count and the next
  // step's (the leader's share of it); read once per step
  struct Step {
    int jm, jm1;
  };
  __device__ __forceinline__ Step step(int t) const { return Step{jmax(t), jmax(t + 1)}; }
  // the leader's tiles of step t + 1, listed at step t
  __device__ __forceinline__ int ahead_count(const Step &s) const { return dQ.div(max(s.jm1 - 1, 0)); }
  // tiles j >= 2 of step t that are not the leader's
  __device__ __forceinline__ int rank_positions(const Step &s) const {
    const int npos = max(s.jm - 1, 0);
    return Q == 0 ? npos : npos - dQ.div(npos);
  }
  // tiles owned by `rank` at a step; D_k is always last, on rank 0
  __device__ __forceinline__ int count(const Step &s) const {
    const int jm = s.jm;
    if (C == 1) return jm + 1;
    if (rank == 0) return (jm >= 1 ? 1 : 0) + (Q == 0 ? 0 : ahead_count(s)) + 1;
    const int N = rank_positions(s);
    return N > rank - 1 ? dC1.div(N - rank) + 1 : 0;
  }
  // j of the idx-th owned tile, in processing order: a rank's tiles j >= 2
  // from the oldest block down; the leader's j = 1 tile, its tiles of step
  // t + 1 from the oldest block down, then D_k (j = 0)
  __device__ __forceinline__ int jat(const Step &s, int idx) const {
    const int jm = s.jm;
    if (C == 1) return idx < jm ? jm - idx : 0;
    if (rank == 0) {
      const int a = jm >= 1 ? 1 : 0;
      if (idx < a) return 1;
      if (Q == 0) return 0;
      const int F1 = ahead_count(s), e = idx - a;
      return e < F1 ? (F1 - 1 - e) * Q + (Q - 1) + 2 : 0;
    }
    const int N = rank_positions(s);
    const int n = N > rank - 1 ? dC1.div(N - rank) + 1 : 0;
    const int i = (rank - 1) + (n - 1 - idx) * (C - 1);
    return (Q == 0 ? i : i + dQ1.div(i)) + 2;
  }
  // whether a tile j at step t is the leader's tile of step t + 1
  __device__ __forceinline__ bool ahead(int j) const { return rank == 0 && C > 1 && Q > 0 && j >= 2; }
};

__device__ __forceinline__ const double *tile_src(const Job &Jb, int t, int j) {
  const int nblk = Jb.nblk;
  const size_t J1 = Jb.J + 1;
  if (t < nblk) {
    const int k = t;
    return j ? Jb.tiles + ((size_t)k * J1 + j) * TSZ : Jb.dinv + (size_t)k * TSZ;
  }
  const int k = 2 * nblk - 1 - t;
  return j ? Jb.tiles + ((size_t)(k + j) * J1 + j) * TSZ : Jb.dinv + (size_t)k * TSZ;
}

// Two CTAs per SM for up to two planes (128 registers a thread), one for more.
template <int PMAX>
__global__ void __launch_bounds__(256, PMAX <= 2 ? 2 : 1)
    k_band_sweep(const Job *__restrict__ jobs, int C, int S, int Wmax, int Q) {
  const int rank = (int)cluster_ctarank();
  const Job Jb = jobs[blockIdx.x / C];
  const int P = Jb.P, nblk = Jb.nblk, W = Jb.J + 2;
  extern __shared__ __align__(128) unsigned char smraw[];
  double *ring = reinterpret_cast<double *>(smraw);      // S * TSZ
  double *ysl = ring + (size_t)S * TSZ;                  // 2 * PMAX * NB: y of this tile and the next
  double *pbuf = ysl + (size_t)2 * PMAX * NB;            // 2 * (C-1) * PMAX * NB
  double *qpart = pbuf + (size_t)2 * max(C - 1, 1) * PMAX * NB;  // 4 * PMAX * NB
  double *acc = qpart + 4 * PMAX * NB;                   // PMAX * NB
  double *yk = acc + PMAX * NB;                          // PMAX * NB
  uint64_t *full = reinterpret_cast<uint64_t *>(yk + PMAX * NB);  // S
  uint64_t *ybar = full + S;                             // Wmax
  uint64_t *pbar = ybar + Wmax;                          // 2
  __shared__ int abort_flag;

  const int tid = threadIdx.x, c = tid & (NB - 1), q = tid >> 6;
  const SweepGeom G{nblk,
                    Jb.J,
                    C,
                    rank,
                    Q,
                    FastDiv((unsigned)max(C - 1, 1)),
                    FastDiv((unsigned)max(Q, 1)),
                    FastDiv((unsigned)max(Q - 1, 1)),
                    Jb.jf,
                    Jb.jb};
  const FastDiv dW((unsigned)W);
  const long long lim = g_sweep_wait;
  if (tid == 0) {
    for (int s = 0; s < S; s++) mbar_init(&full[s], 1);
    for (int w = 0; w < Wmax; w++) mbar_init(&ybar[w], 1);
    mbar_init(&pbar[0], max(C - 1, 1));
    mbar_init(&pbar[1], max(C - 1, 1));
    fence_mbar_init_cluster();
    abort_flag = 0;
  }
  __syncthreads();
  cluster_sync_all();

  const int T = 2 * nblk;
  // producer state (thread 0): next tile (tp, ip); counters are uniform.
  int tp = 0, ip = 0, pslot = 0;
  SweepGeom::Step ps = G.step(0);  // the producer's step tp
  long long nissued = 0, ncons = 0;
  int cslot = 0;
  uint32_t cphase = 0;  // slot and phase parity of tile ncons
  auto consumed = [&]() {
    ncons++;
    if (++cslot == S) {
      cslot = 0;
      cphase ^= 1u;
    }
  };
  auto produce = [&](long long limit) {
    while (nissued < limit) {
      while (tp < T && ip >= G.count(ps)) {
        tp++;
        ip = 0;
        ps = SweepGeom::Step{ps.jm1, G.jmax(tp + 1)};
      }
      if (tp >= T) return;
      const int j = G.jat(ps, ip);
      double *dst = ring + (size_t)pslot * TSZ;
      uint64_t *bar = &full[pslot];
      if (++pslot == S) pslot = 0;
      mbar_arrive_expect_tx(bar, (uint32_t)(TSZ * sizeof(double)));
      // the leader's share is listed a step early: the tile is step tp + 1's
      bulk_g2s(dst, tile_src(Jb, G.ahead(j) ? tp + 1 : tp, j), (uint32_t)(TSZ * sizeof(double)), bar);
      nissued++;
      ip++;
    }
  };
  if (tid == 0) produce(S);

  // Block src (the one solved at step src) from the RHS array into ysl[b]:
  // threads tid < P NB / 2 copy one 16-byte chunk each through L2.
  auto copy_y = [&](int src, int b) {
    if (tid < P * (NB / 2)) {
      const int p = tid / (NB / 2), ch = tid - p * (NB / 2);
      const int blk = src < nblk ? src : 2 * nblk - 1 - src;
      cp_async16_cg(ysl + ((size_t)b * PMAX + p) * NB + 2 * ch,
                    Jb.rhs + (size_t)p * Jb.rhs_stride + (size_t)blk * NB + 2 * ch);
    }
    cp_async_commit();
  };
  // The block a tile (t, j >= 2) multiplies, solved at step t - j (t + 1 - j
  // for the leader's tiles of the next step): every thread of a rank waits
  // (bounded) for the leader's release of it, then copies its chunk.  False
  // if the wait ran out (nothing is copied then).
  auto fetch_y = [&](int t, int j, int b) -> bool {
    const int src = (G.ahead(j) ? t + 1 : t) - j;
    // only the copying threads need the release (the others read the block
    // after a barrier that follows the copies)
    if (rank != 0 && tid < P * (NB / 2)) {
      const int qw = dW.div(src);
      if (!mbar_wait(&ybar[src - qw * W], (uint32_t)(qw & 1), lim)) return false;
    }
    copy_y(src, b);
    return true;
  };
  // Tiles that multiply a fetched block alternate between the two halves of
  // ysl (ytile counts them, the same in every thread).  The next step's
  // first such block is fetched under the current step's last one when its
  // release is already visible to this thread (one probe, no wait): each
  // thread copies its own chunk, so each may decide alone (pre).
  long long ytile = 0;
  bool pre = false;

  // the leader's right-hand side of the next block column, loaded a step
  // ahead (threads q == 0: column c, each plane); the first backward step's
  // is the forward sweep's last block, taken from the registers that solve it
  double bnext[PMAX];
  if (rank == 0 && q == 0) {
#pragma unroll
    for (int p = 0; p < PMAX; p++)
      if (p < P) bnext[p] = Jb.rhs[(size_t)p * Jb.rhs_stride + c];
  }

  // the leader's partial sums of its tiles of the next step (leader share)
  double sn[PMAX];
#pragma unroll
  for (int p = 0; p < PMAX; p++) sn[p] = 0.0;

  for (int t = 0; t < T; t++) {
    const bool fwd = t < nblk;
    const int k = fwd ? t : 2 * nblk - 1 - t;
    const SweepGeom::Step cs = G.step(t);
    const int n = G.count(cs);
    double s[PMAX];
#pragma unroll
    for (int p = 0; p < PMAX; p++) {
      s[p] = sn[p];  // zero unless the leader worked on this step's tiles during the last one
      sn[p] = 0.0;
    }
    bool bad = false;
    // the step's first tile's block; each later one is fetched under the
    // work of the tile before it (j = 1 uses the leader's own yk, D_k none)
    int jn = n > 0 ? G.jat(cs, 0) : 0;
    if (jn >= 2 && !pre && !fetch_y(t, jn, (int)(ytile & 1))) bad = true;
    pre = false;
    for (int idx = 0; idx < n; idx++) {
      const int j = jn;
      if (j == 0) break;  // D_k: handled below by the leader
      const int slot = cslot;
      if (!mbar_wait(&full[slot], cphase, lim)) bad = true;
      cp_async_wait_all();  // this thread's chunks of the tile's block
      if (bad) abort_flag = 1;
      __syncthreads();
      if (abort_flag) break;
      const double *yv = yk;
      if (j >= 2) yv = ysl + (size_t)(ytile++ & 1) * PMAX * NB;
      jn = idx + 1 < n ? G.jat(cs, idx + 1) : 0;
      // ysl[ytile & 1] was last read two fetched tiles ago, before the
      // barrier that ended it; a failed wait is seen after this tile's barrier
      if (jn >= 2) {
        if (!fetch_y(t, jn, (int)(ytile & 1))) abort_flag = 1;
      } else if (t + 1 < T) {
        const SweepGeom::Step ns = SweepGeom::Step{cs.jm1, G.jmax(t + 2)};
        const int n1 = G.count(ns), j1 = n1 > 0 ? G.jat(ns, 0) : 0;
        const int src = (G.ahead(j1) ? t + 2 : t + 1) - j1;
        // the leader copies without a release; block t itself is solved
        // only at the end of this step
        const int qw = dW.div(src);
        if (j1 >= 2 && (rank == 0 ? src < t : mbar_test_cluster(&ybar[src - qw * W], (uint32_t)(qw & 1)))) {
          copy_y(src, (int)(ytile & 1));
          pre = true;
        }
      }
      const double *Tt = ring + (size_t)slot * TSZ;
      // the leader's tiles of the next step go to sn, every other tile to s
      auto tile_dot = [&](double(&acc)[PMAX]) {
        if (fwd) {
#pragma unroll 4
          for (int rr = q * 16; rr < q * 16 + 16; rr++) {
            const double tv = Tt[rr * LDT + c];
#pragma unroll
            for (int p = 0; p < PMAX; p++)
              if (p < P) acc[p] += tv * yv[p * NB + rr];
          }
        } else {
#pragma unroll 4
          for (int cc = q * 16; cc < q * 16 + 16; cc++) {
            const double tv = Tt[c * LDT + cc];
#pragma unroll
            for (int p = 0; p < PMAX; p++)
              if (p < P) acc[p] += tv * yv[p * NB + cc];
          }
        }
      };
      if (G.ahead(j))
        tile_dot(sn);
      else
        tile_dot(s);
      __syncthreads();
      consumed();
      if (tid == 0) produce(ncons + S);
    }
    if (abort_flag) break;
    // reduce the four row quarters in fixed order
#pragma unroll
    for (int p = 0; p < PMAX; p++)
      if (p < P) qpart[(q * PMAX + p) * NB + c] = s[p];
    __syncthreads();
    if (rank != 0) {
      // The leader reads pbuf[t & 1] of step t-2 before it publishes block
      // t-2; seeing that block means the slot is free again.
      if (t >= 2) {
        const int src = t - 2, qw = dW.div(src);
        if (!mbar_wait(&ybar[src - qw * W], (uint32_t)(qw & 1), lim)) abort_flag = 1;
        __syncthreads();
        if (abort_flag) break;
      }
      // partial -> leader's pbuf[t & 1][rank-1]
      if (q == 0) {
        for (int p = 0; p < P; p++) {
          const double v = qpart[(0 * PMAX + p) * NB + c] + qpart[(1 * PMAX + p) * NB + c] +
                           qpart[(2 * PMAX + p) * NB + c] + qpart[(3 * PMAX + p) * NB + c];
          double *dst = pbuf + ((size_t)((t & 1) * (C - 1) + (rank - 1)) * PMAX + p) * NB + c;
          st_cluster_f64(map_rank(dst, 0), v);
        }
        fence_acq_rel_cluster();
      }
      __syncthreads();
      if (tid == 0) mbar_arrive_cluster(map_rank(&pbar[t & 1], 0));
      continue;
    }
    // ---- leader: combine partials, apply D_k, broadcast ----
    if (C > 1) {
      if (!mbar_wait(&pbar[t & 1], (uint32_t)((t >> 1) & 1), lim)) abort_flag = 1;
    }
    if (!mbar_wait(&full[cslot], cphase, lim)) abort_flag = 1;
    __syncthreads();
    if (abort_flag) break;
    if (q == 0) {
#pragma unroll
      for (int p = 0; p < PMAX; p++) {
        if (p >= P) continue;
        double v = qpart[(0 * PMAX + p) * NB + c] + qpart[(1 * PMAX + p) * NB + c] +
                   qpart[(2 * PMAX + p) * NB + c] + qpart[(3 * PMAX + p) * NB + c];
        for (int r = 1; r < C; r++) v += pbuf[((size_t)((t & 1) * (C - 1) + (r - 1)) * PMAX + p) * NB + c];
        acc[p * NB + c] = bnext[p] - v;
      }
    }
    __syncthreads();
    {
      const double *Dk = ring + (size_t)cslot * TSZ;
#pragma unroll
      for (int p = 0; p < PMAX; p++) s[p] = 0.0;
      for (int cc = q * 16; cc < q * 16 + 16; cc++) {
        const double dv = fwd ? Dk[cc * LDT + c] : Dk[c * LDT + cc];
#pragma unroll
        for (int p = 0; p < PMAX; p++)
          if (p < P) s[p] += dv * acc[p * NB + cc];
      }
    }
    __syncthreads();  // all reads of D_k done
    consumed();
    if (tid == 0) produce(ncons + S);
#pragma unroll
    for (int p = 0; p < PMAX; p++)
      if (p < P) qpart[(q * PMAX + p) * NB + c] = s[p];
    __syncthreads();
    if (q == 0) {
#pragma unroll
      for (int p = 0; p < PMAX; p++) {
        if (p >= P) continue;
        const double v = qpart[(0 * PMAX + p) * NB + c] + qpart[(1 * PMAX + p) * NB + c] +
                         qpart[(2 * PMAX + p) * NB + c] + qpart[(3 * PMAX + p) * NB + c];
        yk[p * NB + c] = v;
        Jb.rhs[(size_t)p * Jb.rhs_stride + (size_t)k * NB + c] = v;
        if (t + 1 == nblk) bnext[p] = v;  // backward from the last block: its y is its right-hand side
      }
    }
    // block t is in rhs (and yk): release it to every other rank (slot
    // t % W of their barriers); the writers' fence orders their stores
    // before the arrivals that follow the barrier
    if (q == 0) fence_acq_rel_cluster();
    __syncthreads();
    if (tid > 0 && tid < C) mbar_arrive_cluster(map_rank(&ybar[dW.mod(t)], (uint32_t)tid));
    // the next step's right-hand side, issued after the fence (which would
    // wait for it) and used a step later
    if (q == 0 && t + 1 < T && t + 1 != nblk) {
      const int kn = t + 1 < nblk ? t + 1 : 2 * nblk - 2 - t;  // next step's block column
#pragma unroll
      for (int p = 0; p < PMAX; p++)
        if (p < P) bnext[p] = Jb.rhs[(size_t)p * Jb.rhs_stride + (size_t)kn * NB + c];
    }
  }

  if (abort_flag) {
    cp_async_wait_all();
    if (tid == 0) {
      atomicOr(Jb.status, 1 << SX_ERR_TIMEOUT);
      // drain this CTA's bulk copies still in flight (bounded)
      for (long long i = ncons; i < nissued; i++) {
        mbar_wait(&full[cslot], cphase, WAIT_LIMIT);
        if (++cslot == S) {
          cslot = 0;
          cphase ^= 1u;
        }
      }
    }
    __syncthreads();
  }
  cluster_sync_all();
}

size_t sweep_smem(int pmax, int C, int S, int Wmax) {
  return sizeof(double) * ((size_t)S * TSZ + (size_t)2 * pmax * NB +
                           (size_t)2 * std::max(C - 1, 1) * pmax * NB + 6 * (size_t)pmax * NB) +
         sizeof(uint64_t) * (S + Wmax + 2);
}

// Dynamic shared memory available to the sweep kernels: the opt-in limit
// minus their static shared memory.
static int smem_optin() {
  static int v = 0;
  if (!v) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes a2, a8;
    cudaFuncGetAttributes(&a2, k_band_sweep<2>);
    cudaFuncGetAttributes(&a8, k_band_sweep<8>);
    v = optin - (int)std::max(a2.sharedSizeBytes, a8.sharedSizeBytes);
  }
  return v;
}

// Launch both sweeps for every job: one cluster of sc.C CTAs per job.
int band_sweep_jobs(const Job *djobs, const std::vector<Job> &hjobs, const BandSched &sc, cudaStream_t st) {
  const int C = sc.C, smax = sc.S;
  const int nj = (int)hjobs.size();
  if (nj == 0) return SX_OK;
  int maxP = 0, Wmax = 0;
  for (const Job &j : hjobs) {
    maxP = std::max(maxP, j.P);
    Wmax = std::max(Wmax, j.J + 2);
  }
  if (maxP > 8) return SX_ERR_UNSUPPORTED;
  const int pmax = maxP <= 2 ? 2 : 8;
  const int limit = smem_optin();
  int S = std::max(1, std::min(smax, BAND_STAGES_MAX));
  while (S > 1 && sweep_smem(pmax, C, S, Wmax) > (size_t)limit) S--;
  const size_t sm = sweep_smem(pmax, C, S, Wmax);
  if (sm > (size_t)limit) {
    set_error("band sweep needs %zu B of shared memory (limit %d)", sm, limit);
    return SX_ERR_UNSUPPORTED;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C * nj, 1, 1);
  cfg.blockDim = dim3(256, 1, 1);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (pmax == 2)
    SX_CUDA(cudaLaunchKernelEx(&cfg, k_band_sweep<2>, djobs, C, S, Wmax, std::max(sc.Q, 0)));
  else
    SX_CUDA(cudaLaunchKernelEx(&cfg, k_band_sweep<8>, djobs, C, S, Wmax, std::max(sc.Q, 0)));
  return SX_OK;
}

int prepare_band_kernels() {
  const int limit = smem_optin();
  SX_CUDA(cudaFuncSetAttribute(k_band_sweep<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit));
  SX_CUDA(cudaFuncSetAttribute(k_band_sweep<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit));
  SX_CUDA(cudaFuncSetAttribute(k_band_sweep<2>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  SX_CUDA(cudaFuncSetAttribute(k_band_sweep<8>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  return SX_OK;
}

int default_lead(int C, int J) {
  // an equal share (the last of every C positions) was the fastest share on
  // every cluster size measured (config-3 band, 64 systems: C = 2, 3, 4);
  // with fewer than C positions per block column the leader gets none
  return (C >= 2 && J - 1 >= C) ? C : 0;
}

// Largest cluster size (<= cmax) for which `nj` clusters can be resident at
// once; at least 1.
int band_active_clusters(int C, int pmax, int Wmax, int smax) {
  int S = std::max(1, std::min(smax, BAND_STAGES_MAX));
  while (S > 1 && sweep_smem(pmax, C, S, Wmax) > (size_t)smem_optin()) S--;
  if (sweep_smem(pmax, C, S, Wmax) > (size_t)smem_optin()) return 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C, 1, 1);
  cfg.blockDim = dim3(256, 1, 1);
  cfg.dynamicSmemBytes = sweep_smem(pmax, C, S, Wmax);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  const cudaError_t e = pmax == 2 ? cudaOccupancyMaxActiveClusters(&n, k_band_sweep<2>, &cfg)
                                  : cudaOccupancyMaxActiveClusters(&n, k_band_sweep<8>, &cfg);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// Largest cluster size C <= cmax (and ring depth) for which all nj clusters
// are resident at once, over the ring depths 4, 2 and 1 (a shallower ring
// shrinks a CTA's shared memory, so that two share an SM); the deeper ring
// on a tie.  Depth 1 puts the leader's load of D_k on each block column's
// critical path; it is taken only where the deeper rings leave at most 2
// CTAs per system resident (measured at 4 CTAs on 64 systems with a 37-tile
// band: depth 2, two CTAs per SM, 46 ms; depth 1 61 ms; and at 8 CTAs on 32
// systems with a 17-tile band: depth 2 2.9 ms, depth 1 3.1 ms).
// stages_forced > 0 fixes the depth.
int pick_cluster(int nj, int cmax, int pmax, int Wmax, int *stages_out, int stages_forced) {
  int bestC = 1, bestS = BAND_STAGES_MAX;
  for (int S0 : {BAND_STAGES_MAX, 3, 2, 1}) {
    if (stages_forced > 0 && S0 != stages_forced) continue;
    if (S0 == 1 && stages_forced != 1 && bestC > 2) continue;
    for (int C = 1; C <= cmax; C++) {
      int S = S0;
      while (S > 1 && sweep_smem(pmax, C, S, Wmax) > (size_t)smem_optin()) S--;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(C * nj, 1, 1);
      cfg.blockDim = dim3(256, 1, 1);
      cfg.dynamicSmemBytes = sweep_smem(pmax, C, S, Wmax);
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = C;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int n = 0;
      const cudaError_t e = pmax == 2 ? cudaOccupancyMaxActiveClusters(&n, k_band_sweep<2>, &cfg)
                                      : cudaOccupancyMaxActiveClusters(&n, k_band_sweep<8>, &cfg);
      if (e != cudaSuccess) {
        cudaGetLastError();
        continue;
      }
      if (n >= nj && C > bestC) {
        bestC = C;
        bestS = S0;
      }
    }
  }
  if (stages_forced > 0) bestS = stages_forced;
  if (stages_out) *stages_out = bestS;
  return bestC;
}

}  // namespace sx
