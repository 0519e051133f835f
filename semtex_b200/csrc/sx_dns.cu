// sx_dns.cu -- the field operations of the DNS elliptic phase that build the
// Helmholtz solves' forcing and consume their solutions, on device planes in
// the solve entry points' layout (nz planes plane_stride doubles apart; each
// plane element-major, each element np x np row-major).
//
// Reference:
//   AuxField::gradient      src/auxfield.cpp:514-616 (the scalar branch, :583-612)
//   Element::grad           src/element.cpp:552-596
//   inverse partials        src/element.cpp:1403-1411, null mapping :1431-1434
//   waveProp                dns/integrate.cpp:227-259
//   setPForce               dns/integrate.cpp:262-277
//   project                 dns/integrate.cpp:280-310
//   Field::smooth           src/field.cpp:190-276
//   Element::bndryDsSum     src/element.cpp:464-487, bndryInsert :540-548
//   Integration::StifflyStable / Extrapolation  src/integration.cpp:98-163
//
// Every operation is bound by HBM traffic: each field plane is read once and
// each result written once; the per-element partials are read once per CTA
// and reused over a group of planes.
#include <algorithm>

#include "sx_internal.h"
#include "sx_modal.h"
#include "sx_ptx.cuh"

namespace sx {
namespace {

// ---------------------------------------------------------------------------
// element kernels: x / y derivatives (Element::grad) with their epilogues
// ---------------------------------------------------------------------------
//
// A CTA holds a tile of TE consecutive elements of one plane in shared
// memory and walks a group of planes, copying the next planes' tiles in
// (a cp.async ring) while it works on this one.  It has a group of 64 "row"
// threads and a group of 64 "column" threads.  Row thread (t, r) forms row r
// of element t's r-derivative,
//     dr[r][j] = sum_k u[r][k] D[j][k]        (u D^T, src/element.cpp:569)
// times that row of dr/dx (or dr/dy) into A; column thread (t, c) forms
// column c of the s-derivative,
//     ds[i][c] = sum_k D[i][k] u[k][c]        (D u, src/element.cpp:570)
// times ds/dx (or ds/dy) into C.  Where an operation forms two derivatives
// (a "job" each: pressure forcing's d/dx u and d/dy v, project's d/dx P and
// d/dy P), a thread forms both for its line.  The epilogue adds C + A --
// the rounding sequence of vmul + vvtvp (src/element.cpp:571-572) -- and
// applies the operation's own arithmetic on the way out.  D is a kernel
// parameter: every thread of a warp reads the same entry at the same time,
// so it is a constant-bank operand of the FMA; each thread keeps its row
// (column) of each job's partial in registers for the whole plane group.

constexpr int EL_GROUP = 64;

enum ElemOp { OP_GRAD = 0, OP_PFORCE = 1, OP_PROJECT = 2 };

template <int NP>
struct DMat {
  double d[NP * NP];
};

template <int NP>
constexpr int tile_elems() {
  return EL_GROUP / NP;
}
// odd row pitch: the row walks (stride LP) and the column walks (stride 1)
// of a warp are free of bank conflicts
template <int NP>
constexpr int row_pitch() {
  return NP | 1;
}
template <int NP>
constexpr int tile_words() {
  return tile_elems<NP>() * NP * row_pitch<NP>();
}
// a staged field's slot: the tile rounded up to 16 bytes
template <int NP>
constexpr int stage_words() {
  return (tile_words<NP>() + 1) & ~1;
}
// fields staged per plane, at most: GRAD u; PFORCE u, v and w's partner
// plane; PROJECT P and P's partner plane (its u^ components go straight to
// registers: only the epilogue reads them)
template <int OP>
constexpr int max_stage() {
  return OP == OP_GRAD ? 1 : OP == OP_PFORCE ? 3 : 2;
}
template <int OP>
constexpr int n_jobs() {
  return OP == OP_GRAD ? 1 : 2;  // derivatives formed per plane
}
// planes in the copy ring: two in flight while a third is worked on
template <int OP>
constexpr int el_ring() {
  return 3;
}
// product arrays a line thread writes: project keeps its x and y
// derivatives apart; pressure forcing needs only their sum
template <int OP>
constexpr int n_prod() {
  return OP == OP_PROJECT ? 2 : 1;
}
// tiles [ring slots][staged fields], then A [products], C [products]
template <int NP, int OP>
constexpr size_t elem_smem(int nstage) {
  return sizeof(double) *
         ((size_t)el_ring<OP>() * nstage * stage_words<NP>() + 2 * n_prod<OP>() * tile_words<NP>());
}
// a row group and a column group; with two jobs a thread forms both, each
// D entry it reads serving two multiply-adds
template <int OP>
constexpr int elem_threads() {
  return 2 * EL_GROUP;
}
template <int OP>
constexpr int elem_min_blocks() {
  return OP == OP_GRAD ? 6 : 3;
}

struct ElemArgs {
  // fields staged into shared memory plane by plane; a "partner" field is
  // read at plane z ^ 1 (the other half of plane z's Fourier mode)
  const double *stage[6];
  int partner[6];
  int nstage;
  const double *us[4];    // PROJECT: u^ components
  double *out;            // GRAD: the field itself (in place); PFORCE: the forcing
  double *uf[4];          // PROJECT: results
  // partials of job 0 (r, s) and job 1 (r, s)
  const double *r0, *s0, *r1, *s1;
  long long stride;
  int nel, nz, zgroup, base, ndim, ncom, nadv;
  double beta, dtinv, alpha, bvisc, prandtl;
};

// Row r of a tile times D^T (row threads) or D times column r (column
// threads), scaled by the thread's partials p: into dst at the same places.
template <int NP, int LP>
__device__ __forceinline__ void deriv_line(const double *__restrict__ T, double *__restrict__ dst, bool rowt, int t,
                                           int r, const DMat<NP> &D, const double (&p)[NP]) {
  const int b = rowt ? (t * NP + r) * LP : t * NP * LP + r;
  const int step = rowt ? 1 : LP;
  double u[NP];
#pragma unroll
  for (int k = 0; k < NP; k++) u[k] = T[b + k * step];
#pragma unroll
  for (int j = 0; j < NP; j++) {
    double d = 0.0;
#pragma unroll
    for (int k = 0; k < NP; k++) d = fma(u[k], D.d[j * NP + k], d);
    dst[b + j * step] = __dmul_rn(d, p[j]);
  }
}

// Both jobs of a line: two fields with a partial each (TWO_FIELDS: u's
// x-product plus v's y-product, summed into d0) or one field with two
// partials (the x and y derivatives of the same P, into d0 and d1).
template <int NP, int LP, bool TWO_FIELDS>
__device__ __forceinline__ void deriv_pair(const double *__restrict__ T0, const double *__restrict__ T1,
                                           double *__restrict__ d0, double *__restrict__ d1, bool rowt, int t,
                                           int r, const DMat<NP> &D, const double (&p0)[NP],
                                           const double (&p1)[NP]) {
  const int b = rowt ? (t * NP + r) * LP : t * NP * LP + r;
  const int step = rowt ? 1 : LP;
  double u[NP], v[NP];
#pragma unroll
  for (int k = 0; k < NP; k++) {
    u[k] = T0[b + k * step];
    v[k] = TWO_FIELDS ? T1[b + k * step] : 0.0;
  }
#pragma unroll
  for (int j = 0; j < NP; j++) {
    double x = 0.0, y = 0.0;
#pragma unroll
    for (int k = 0; k < NP; k++) {
      const double dk = D.d[j * NP + k];
      x = fma(u[k], dk, x);
      if (TWO_FIELDS) y = fma(v[k], dk, y);
    }
    if (TWO_FIELDS) {
      d0[b + j * step] = __dadd_rn(__dmul_rn(x, p0[j]), __dmul_rn(y, p1[j]));
    } else {
      d0[b + j * step] = __dmul_rn(x, p0[j]);
      d1[b + j * step] = __dmul_rn(x, p1[j]);
    }
  }
}

template <int NP, int OP>
__global__ void __launch_bounds__(elem_threads<OP>(), elem_min_blocks<OP>())
    k_elem(const ElemArgs a, const DMat<NP> D) {
  constexpr int TE = tile_elems<NP>(), LP = row_pitch<NP>(), TW = tile_words<NP>(), SW = stage_words<NP>();
  constexpr int NS = max_stage<OP>(), NJ = n_jobs<OP>(), NT = elem_threads<OP>();
  constexpr bool FLAT = LP == NP;  // tile rows unpadded: the tile is the plane's contiguous run
  constexpr int EL_RING = el_ring<OP>();
  extern __shared__ __align__(16) double sm[];
  const int ns = a.nstage;
  double *tiles = sm;                  // [EL_RING buffers][ns][SW]
  double *A = sm + EL_RING * ns * SW;  // [n_prod][TW] row products
  double *Cs = A + n_prod<OP>() * TW;  // [n_prod][TW] column products
  const int tid = threadIdx.x;
  const int e0 = blockIdx.x * TE;
  const int ne = min(TE, a.nel - e0);
  const int nwords = ne * NP * NP;  // the tile's contiguous doubles in a plane
  const int z0 = blockIdx.y * a.zgroup, z1 = min(a.nz, z0 + a.zgroup);
  const bool rowt = tid < EL_GROUP;
  const int lt = rowt ? tid : tid - EL_GROUP;
  const int t = lt / NP, r = lt - (lt / NP) * NP;
  const bool active = t < ne;

  // this thread's row (row threads) or column (column threads) of each
  // job's partial
  double p0[NP], p1[NP];
  {
    const double *q0 = rowt ? a.r0 : a.s0, *q1 = rowt ? a.r1 : a.s1;
    const size_t eb = (size_t)(e0 + (active ? t : 0)) * NP * NP;
#pragma unroll
    for (int k = 0; k < NP; k++) {
      const size_t node = eb + (rowt ? r * NP + k : k * NP + r);
      p0[k] = active ? q0[node] : 0.0;
      p1[k] = (NJ == 2 && active) ? q1[node] : 0.0;
    }
  }
  double *prod = rowt ? A : Cs;

  // every call commits one cp.async group (empty past the plane group's
  // end), so that "all but the newest EL_RING - 1 groups" is always plane z
  auto issue = [&](int z, int buf) {
#pragma unroll
    for (int f = 0; f < NS; f++) {
      if (f >= ns || z >= z1) break;
      const double *src = a.stage[f] + (size_t)(a.partner[f] ? z ^ 1 : z) * a.stride + (size_t)e0 * NP * NP;
      double *dst = tiles + (buf * ns + f) * SW;
      if (FLAT) {
        for (int i = tid; i < nwords; i += NT) cp_async8_ca(dst + i, src + i);
      } else {
        for (int i = tid; i < nwords; i += NT) {
          const int row = i / NP;
          cp_async8_ca(dst + row * LP + (i - row * NP), src + i);
        }
      }
    }
    cp_async_commit();
  };

  for (int q = 0; q < EL_RING - 1; q++) issue(z0 + q, q);
  for (int z = z0; z < z1; z++) {
    const int buf = (z - z0) % EL_RING;
    // the ring slot of plane z + EL_RING - 1 was last read in iteration z - 1,
    // which every thread has left (the barrier that ends it)
    issue(z + EL_RING - 1, (buf + EL_RING - 1) % EL_RING);
    cp_async_wait_ring<EL_RING - 1>();
    __syncthreads();
    auto S = [&](int f) { return tiles + (buf * ns + f) * SW; };
    // project's u^ values at this thread's epilogue points, loaded now so
    // that they arrive while the derivatives are formed
    constexpr int NI = OP == OP_PROJECT ? (TE * NP * NP + NT - 1) / NT : 1;
    double ur[NI][4];
    if (OP == OP_PROJECT) {
      const size_t pz = (size_t)z * a.stride + (size_t)e0 * NP * NP;
#pragma unroll
      for (int q = 0; q < NI; q++) {
        const int i = tid + q * NT;
#pragma unroll
        for (int c = 0; c < 4; c++) ur[q][c] = (i < nwords && c < a.nadv) ? a.us[c][pz + i] : 0.0;
      }
    }
    if (active) {
      if (OP == OP_GRAD)
        deriv_line<NP, LP>(S(0), prod, rowt, t, r, D, p0);
      else
        deriv_pair<NP, LP, OP == OP_PFORCE>(S(0), S(1), prod, prod + TW, rowt, t, r, D, p0, p1);
    }
    __syncthreads();
    // d/dz factor of plane z (src/auxfield.cpp:597-610): mode k = z/2 + base;
    // Re' = -beta k Im, Im' = beta k Re; zero for mode 0 and Nyquist when base is 0
    const int kz = (z >> 1) + a.base;
    const double bz = (a.base == 0 && z < 2) ? 0.0 : ((z & 1) ? a.beta * (double)kz : -(a.beta * (double)kz));
    // epilogue, coalesced over the tile's doubles of plane z
    const size_t pb = (size_t)z * a.stride + (size_t)e0 * NP * NP;
    const double *sz = OP == OP_PFORCE ? S(ns == 3 ? 2 : 0) : S(a.ndim == 3 ? 1 : 0);  // the z partner
#pragma unroll
    for (int q = 0; q < (OP == OP_PROJECT ? NI : (TE * NP * NP + NT - 1) / NT); q++) {
      const int i = tid + q * NT;
      if (i >= nwords) break;
      const int si = FLAT ? i : (i / NP) * LP + (i - (i / NP) * NP);
      const size_t gi = pb + i;
      const double g0 = __dadd_rn(Cs[si], A[si]);
      if (OP == OP_GRAD) {
        a.out[gi] = g0;
      } else if (OP == OP_PFORCE) {
        // ((d/dx u + d/dy v) + d/dz w) / dt  (dns/integrate.cpp:272-276); the
        // four derivative products are summed as (s terms) + (r terms), each
        // pair added where it is formed, so each takes one trip through
        // shared memory
        double s = g0;
        if (ns == 3) s = __dadd_rn(s, __dmul_rn(bz, sz[si]));
        a.out[gi] = __dmul_rn(s, a.dtinv);
      } else {
        // u^^ = alpha u^ (times Pr for the scalar) + bvisc grad P
        // (dns/integrate.cpp:296-309); staged: P, P's partner, u^ ...
        const double g1 = __dadd_rn(Cs[TW + si], A[TW + si]);
#pragma unroll
        for (int c = 0; c < 4; c++) {
          if (c >= a.nadv) break;
          double v = __dmul_rn(a.alpha, ur[OP == OP_PROJECT ? q : 0][c]);
          if (c == a.ncom) v = __dmul_rn(v, a.prandtl);
          if (c < a.ndim) {
            const double g = c == 0 ? g0 : c == 1 ? g1 : __dmul_rn(bz, sz[si]);
            v = __dadd_rn(v, __dmul_rn(a.bvisc, g));
          }
          a.uf[c][gi] = v;
        }
      }
    }
    __syncthreads();
  }
}

// d/dz in place on Fourier planes (src/auxfield.cpp:597-610): thread per
// (mode, point), both planes of the mode read before either is written.
__global__ void k_dz_inplace(double *__restrict__ w, int nmodes, int npts, long long stride, int base, double beta) {
  const int m = blockIdx.y;
  double *re = w + (size_t)(2 * m) * stride, *im = re + stride;
  const int k = m + base;
  const double bk = beta * (double)k;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += gridDim.x * blockDim.x) {
    if (base == 0 && m == 0) {
      re[i] = 0.0;
      im[i] = 0.0;
    } else {
      const double a = re[i], b = im[i];
      re[i] = __dmul_rn(-bk, b);
      im[i] = __dmul_rn(bk, a);
    }
  }
}

// ---------------------------------------------------------------------------
// Field::smooth: mass-weighted direct stiffness average of element boundaries
// ---------------------------------------------------------------------------
//
// Thread per global node g.  The reference sums Q4 u of every element slot
// holding g into dssum[g] element after element, scales by imass[g] and
// writes the value back into those slots.  The CSR g2e lists each node's
// slots in element order, so the sum here is the reference's sum, rounding
// for rounding, and each slot is read and written by one thread only.
constexpr int SMOOTH_CACHE = 4;  // holders kept in registers; more are walked in the CSR

__global__ void __launch_bounds__(256, 3)
    k_smooth(double *__restrict__ u, const int *__restrict__ ptr, const int *__restrict__ idx,
             const int *__restrict__ emap, const double *__restrict__ Q4, const double *__restrict__ imass,
             int nglobal, int next, int npnp, int nz, int zgroup, long long stride) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nglobal) return;
  const int z0 = blockIdx.y * zgroup, z1 = min(nz, z0 + zgroup);
  const int b = ptr[g], n = ptr[g + 1] - b;
  int off[SMOOTH_CACHE];
  double wq[SMOOTH_CACHE];
#pragma unroll
  for (int c = 0; c < SMOOTH_CACHE; c++) {
    off[c] = 0;
    wq[c] = 0.0;
    if (c < n) {
      const int slot = idx[b + c], e = slot / next;
      off[c] = e * npnp + emap[slot - e * next];
      wq[c] = Q4[off[c]];
    }
  }
  const double im = imass[g];
  auto dssum = [&](const double *p) {
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < SMOOTH_CACHE; c++)
      if (c < n) s = __dadd_rn(s, __dmul_rn(wq[c], p[off[c]]));
    for (int c = SMOOTH_CACHE; c < n; c++) {  // vertices shared by more elements
      const int slot = idx[b + c], e = slot / next;
      const int o = e * npnp + emap[slot - e * next];
      s = __dadd_rn(s, __dmul_rn(Q4[o], p[o]));
    }
    return __dmul_rn(s, im);
  };
  auto insert = [&](double *p, double s) {
#pragma unroll
    for (int c = 0; c < SMOOTH_CACHE; c++)
      if (c < n) p[off[c]] = s;
    for (int c = SMOOTH_CACHE; c < n; c++) {
      const int slot = idx[b + c], e = slot / next;
      p[e * npnp + emap[slot - e * next]] = s;
    }
  };
  // two planes at a time: both sums' loads are in flight before either
  // plane is written
  int z = z0;
  for (; z + 1 < z1; z += 2) {
    double *p0 = u + (size_t)z * stride, *p1 = p0 + stride;
    const double s0 = dssum(p0), s1 = dssum(p1);
    insert(p0, s0);
    insert(p1, s1);
  }
  if (z < z1) {
    double *p0 = u + (size_t)z * stride;
    insert(p0, dssum(p0));
  }
}

// ---------------------------------------------------------------------------
// waveProp: u^ = sum_q (-alpha_{q+1} u_q + dt beta_q N_q)
// ---------------------------------------------------------------------------

struct WaveArgs {
  const double *us[3][4], *uf[3][4];
  double *h[4];
  double a[3], b[3];  // -alpha_{q+1}, dt beta_q
  int order, nadv;
  long long n;
};

__global__ void __launch_bounds__(256) k_wave_prop(const WaveArgs w) {
  const long long step = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < w.n; i += step)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      if (c >= w.nadv) break;
      // H = 0, then axpy(-alpha[q+1], Us[q]), axpy(beta[q], Uf[q]) level by
      // level (dns/integrate.cpp:241-258)
      double h = 0.0;
#pragma unroll
      for (int q = 0; q < 3; q++) {
        if (q >= w.order) break;
        h = __dadd_rn(h, __dmul_rn(w.a[q], w.us[q][c][i]));
        h = __dadd_rn(h, __dmul_rn(w.b[q], w.uf[q][c][i]));
      }
      w.h[c][i] = h;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

#define SX_DNS_NP_SWITCH(np, CALL)                    \
  switch (np) {                                       \
    case 3: { constexpr int N_ = 3; CALL; } break;   \
    case 4: { constexpr int N_ = 4; CALL; } break;   \
    case 5: { constexpr int N_ = 5; CALL; } break;   \
    case 6: { constexpr int N_ = 6; CALL; } break;   \
    case 7: { constexpr int N_ = 7; CALL; } break;   \
    case 8: { constexpr int N_ = 8; CALL; } break;   \
    case 9: { constexpr int N_ = 9; CALL; } break;   \
    case 10: { constexpr int N_ = 10; CALL; } break; \
    case 11: { constexpr int N_ = 11; CALL; } break; \
    case 12: { constexpr int N_ = 12; CALL; } break; \
    default: return SX_ERR_UNSUPPORTED;               \
  }

// Planes per CTA: as many as keep at least ~4 waves of two CTAs per SM.
int plane_group(long long tiles, int nz) {
  for (int zg : {16, 8, 4, 2})
    if (tiles * ((nz + zg - 1) / zg) >= 4LL * 2 * 148) return std::min(zg, nz);
  return 1;
}

template <int NP, int OP>
int launch_elem(const sx_mesh_s &M, ElemArgs a, cudaStream_t st) {
  constexpr int TE = tile_elems<NP>();
  static_assert(elem_smem<NP, OP>(max_stage<OP>()) <= 227 * 1024, "element tiles do not fit in shared memory");
  const size_t smem = elem_smem<NP, OP>(a.nstage);
  if (smem > 48 * 1024)
    SX_CUDA(cudaFuncSetAttribute(k_elem<NP, OP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  DMat<NP> D;
  for (int i = 0; i < NP * NP; i++) D.d[i] = M.D[i];
  const long long tiles = (M.nel + TE - 1) / TE;
  a.nel = M.nel;
  a.zgroup = plane_group(tiles, a.nz);
  const dim3 grid((unsigned)tiles, (unsigned)((a.nz + a.zgroup - 1) / a.zgroup));
  k_elem<NP, OP><<<grid, elem_threads<OP>(), smem, st>>>(a, D);
  SX_CUDA(cudaGetLastError());
  return SX_OK;
}

template <int OP>
int run_elem(const sx_mesh_s &M, const ElemArgs &a, cudaStream_t st) {
  SX_DNS_NP_SWITCH(M.np, return (launch_elem<N_, OP>(M, a, st)));
  return SX_ERR_UNSUPPORTED;
}

int check_planes(const sx_mesh_s &M, int nz, int plane_stride, const char *who) {
  if (nz < 1 || plane_stride < M.nel * M.npnp) {
    set_error("%s: nz = %d, plane_stride = %d (a plane holds %d points)", who, nz, plane_stride, M.nel * M.npnp);
    return SX_ERR_ARG;
  }
  return check_mesh_device(M, who);
}

}  // namespace
}  // namespace sx

using namespace sx;

extern "C" int sx_field_gradient(sx_mesh mesh, double *d_data, int nz, int plane_stride, int dir, double beta,
                                 int base_mode, void *stream) {
  if (!mesh || !d_data || dir < 0 || dir > 2 || base_mode < 0) return SX_ERR_ARG;
  SX_TRY(check_planes(*mesh, nz, plane_stride, "sx_field_gradient"));
  cudaStream_t st = (cudaStream_t)stream;
  if (dir == 2) {
    if (nz % 2) {
      set_error("sx_field_gradient: d/dz needs Fourier planes in pairs (nz = %d)", nz);
      return SX_ERR_ARG;
    }
    const int npts = mesh->nel * mesh->npnp;
    const dim3 grid((unsigned)std::min((npts + 255) / 256, 148 * 4), (unsigned)(nz / 2));
    k_dz_inplace<<<grid, 256, 0, st>>>(d_data, nz / 2, npts, plane_stride, base_mode, beta);
    SX_CUDA(cudaGetLastError());
    return SX_OK;
  }
  ElemArgs a{};
  a.stage[0] = d_data;
  a.nstage = 1;
  a.out = d_data;
  a.r0 = dir == 0 ? mesh->ddrdx.p : mesh->ddrdy.p;
  a.s0 = dir == 0 ? mesh->ddsdx.p : mesh->ddsdy.p;
  a.r1 = a.r0;
  a.s1 = a.s0;
  a.stride = plane_stride;
  a.nz = nz;
  return run_elem<OP_GRAD>(*mesh, a, st);
}

extern "C" int sx_dns_pressure_forcing(sx_mesh mesh, const double *const *d_us, int ndim, double *d_out, int nz,
                                       int plane_stride, double dt, double beta, int base_mode, void *stream) {
  if (!mesh || !d_us || !d_out || ndim < 2 || ndim > 3 || base_mode < 0) return SX_ERR_ARG;
  for (int i = 0; i < ndim; i++)
    if (!d_us[i]) return SX_ERR_ARG;
  if (dt == 0.0) {
    set_error("sx_dns_pressure_forcing: divide by zero (dt = 0)");
    return SX_ERR_ARG;
  }
  SX_TRY(check_planes(*mesh, nz, plane_stride, "sx_dns_pressure_forcing"));
  if (ndim == 3 && (nz % 2 || d_out == d_us[2])) {
    set_error("sx_dns_pressure_forcing: 3 dimensions need Fourier planes in pairs and an output apart from w");
    return SX_ERR_ARG;
  }
  ElemArgs a{};
  a.stage[0] = d_us[0];
  a.stage[1] = d_us[1];
  if (ndim == 3) {
    a.stage[2] = d_us[2];  // read at each plane's partner: the other half of its mode
    a.partner[2] = 1;
  }
  a.nstage = ndim;
  a.out = d_out;
  a.r0 = mesh->ddrdx.p;
  a.s0 = mesh->ddsdx.p;
  a.r1 = mesh->ddrdy.p;
  a.s1 = mesh->ddsdy.p;
  a.stride = plane_stride;
  a.nz = nz;
  a.ndim = ndim;
  a.base = base_mode;
  a.beta = beta;
  a.dtinv = 1.0 / dt;
  return run_elem<OP_PFORCE>(*mesh, a, (cudaStream_t)stream);
}

extern "C" int sx_dns_project(sx_mesh mesh, const double *const *d_us, const double *d_p, double *const *d_uf,
                              int ndim, int ncom, int nadv, int nz, int plane_stride, double dt, double kinvis,
                              double prandtl, double beta, int base_mode, void *stream) {
  if (!mesh || !d_us || !d_p || !d_uf || ndim < 2 || ndim > 3 || ncom < ndim || ncom > 3 || nadv < ncom ||
      nadv > ncom + 1 || base_mode < 0)
    return SX_ERR_ARG;
  for (int i = 0; i < nadv; i++)
    if (!d_us[i] || !d_uf[i] || d_uf[i] == d_p) return SX_ERR_ARG;
  if (dt * kinvis == 0.0 || kinvis == 0.0) {
    set_error("sx_dns_project: D_T * KINVIS and KINVIS must be nonzero");
    return SX_ERR_ARG;
  }
  SX_TRY(check_planes(*mesh, nz, plane_stride, "sx_dns_project"));
  if (ndim == 3 && nz % 2) {
    set_error("sx_dns_project: 3 dimensions need Fourier planes in pairs (nz = %d)", nz);
    return SX_ERR_ARG;
  }
  ElemArgs a{};
  a.stage[0] = d_p;
  a.nstage = 1;
  if (ndim == 3) {  // P at each plane's partner, for d/dz
    a.stage[1] = d_p;
    a.partner[1] = 1;
    a.nstage = 2;
  }
  for (int i = 0; i < nadv; i++) {
    a.us[i] = d_us[i];
    a.uf[i] = d_uf[i];
  }
  a.r0 = mesh->ddrdx.p;
  a.s0 = mesh->ddsdx.p;
  a.r1 = mesh->ddrdy.p;
  a.s1 = mesh->ddsdy.p;
  a.stride = plane_stride;
  a.nz = nz;
  a.ndim = ndim;
  a.ncom = nadv > ncom ? ncom : -1;  // the scalar's index, when there is one
  a.nadv = nadv;
  a.base = base_mode;
  a.beta = beta;
  a.alpha = -1.0 / (dt * kinvis);
  a.bvisc = 1.0 / kinvis;
  a.prandtl = prandtl;
  return run_elem<OP_PROJECT>(*mesh, a, (cudaStream_t)stream);
}

extern "C" int sx_field_smooth(sx_mesh mesh, double *d_data, int nz, int plane_stride, void *stream) {
  if (!mesh || !d_data) return SX_ERR_ARG;
  SX_TRY(check_planes(*mesh, nz, plane_stride, "sx_field_smooth"));
  const int threads = 256;
  const long long blocks = (mesh->nglobal + threads - 1) / threads;
  const int zg = plane_group(blocks, nz);
  const dim3 grid((unsigned)blocks, (unsigned)((nz + zg - 1) / zg));
  k_smooth<<<grid, threads, 0, (cudaStream_t)stream>>>(d_data, mesh->dg2e_ptr.p, mesh->dg2e_idx.p, mesh->demap.p,
                                                       mesh->dQ4.p, mesh->dimass.p, mesh->nglobal, mesh->next,
                                                       mesh->npnp, nz, zg, plane_stride);
  SX_CUDA(cudaGetLastError());
  return SX_OK;
}

extern "C" int sx_dns_wave_prop(const double *const *d_us, const double *const *d_uf, double *const *d_h, int nadv,
                                int order, long long npts, double dt, void *stream) {
  if (!d_us || !d_uf || !d_h || nadv < 1 || nadv > 4 || order < 1 || order > 3 || npts < 0) return SX_ERR_ARG;
  // Stiffly-stable (backward differentiation) and extrapolation weights of
  // order 1-3 (Gear 1971, Table 11.1; src/integration.cpp:98-163)
  static const double alpha[3][4] = {{1.0, -1.0, 0.0, 0.0}, {1.5, -2.0, 0.5, 0.0}, {11.0 / 6.0, -3.0, 1.5, -1.0 / 3.0}};
  static const double extrap[3][3] = {{1.0, 0.0, 0.0}, {2.0, -1.0, 0.0}, {3.0, -3.0, 1.0}};
  WaveArgs w{};
  for (int q = 0; q < order; q++) {
    w.a[q] = -alpha[order - 1][q + 1];
    w.b[q] = extrap[order - 1][q] * dt;
    for (int c = 0; c < nadv; c++) {
      w.us[q][c] = d_us[q * nadv + c];
      w.uf[q][c] = d_uf[q * nadv + c];
      if (!w.us[q][c] || !w.uf[q][c]) return SX_ERR_ARG;
    }
  }
  for (int c = 0; c < nadv; c++) {
    if (!d_h[c]) return SX_ERR_ARG;
    w.h[c] = d_h[c];
  }
  w.order = order;
  w.nadv = nadv;
  w.n = npts;
  if (npts == 0) return SX_OK;
  const long long blocks = std::min<long long>((npts + 255) / 256, 148LL * 8);
  k_wave_prop<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(w);
  SX_CUDA(cudaGetLastError());
  return SX_OK;
}
