// sx_static.cu -- sx_field_solve_device_static: the plain FP64 direct solve
// (sx_field_solve_device on DIRECT systems) with its per-call scratch in a
// file-scope device array instead of the modal system's grow-only workspace,
// so that a call allocates no device memory.
//
// Callers that cannot allocate: a time-stepping loop whose device memory is
// already held by another allocator (a framework's caching pool sized to the
// card), where cudaMalloc would fail mid-run; and latency-bound loops, where
// the device-wide synchronisation that cudaFree implies would stall every
// other stream.  The first call on a device must have allocated nothing
// either, so the workspace cannot simply be sized on first use there.
//
// The scratch is one array per device, shared by every call: calls that
// overlap in time (two host threads, or two streams) race on it and must be
// serialised by the caller.  Calls enqueued on one stream are ordered by the
// stream and do not race.
#include <cstring>
#include <mutex>

#include "sx_modal.h"

using namespace sx;

// SX_STATIC_SCRATCH_BYTES (4 MiB): one mode (two planes) of a 32 x 32
// element, N = 8 mesh needs about 0.9 MB; 64 x 64 elements at N = 8 about
// 3.5 MB.
static __device__ __align__(256) unsigned char g_scratch[SX_STATIC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void *g_scratch_ptr[kMaxDevices] = {};

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Device address of g_scratch on the current device.  The first call on a
// device looks it up with cudaGetSymbolAddress (which may load this module);
// later calls reuse the cached address.
int scratch_on_current_device(void **out) {
  int dev = 0;
  SX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("sx_field_solve_device_static: device %d outside the %d devices it tracks", dev, kMaxDevices);
    return SX_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) {
      set_error("sx_field_solve_device_static: cudaGetSymbolAddress(scratch) on device %d: %s", dev,
                cudaGetErrorString(e));
      return SX_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return SX_OK;
}

// Plane group g of an nz-plane field (src/field.cpp:564-573): local mode l
// owns planes 2l, 2l+1; plane 1 is the Nyquist datum when the base mode is 0.
struct PlaneGroup {
  int mode, plane0, P;
};

PlaneGroup plane_group(int base_mode, int nz, int l) {
  if (nz == 1 || (l == 0 && base_mode == 0)) return {0, 0, 1};
  return {l, 2 * l, 2};
}

// Stores one mode's job record into the scratch array.  The record travels
// as a kernel argument, which the runtime copies when the launch is
// enqueued, so the host record can be rewritten for the next mode at once
// (a pageable host-to-device copy would instead be read whenever the
// runtime gets to it).
__global__ void k_put_job(Job *dst, Job j) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst = j;
}

}  // namespace

extern "C" int sx_field_solve_device_static(sx_modal s, double *d_u, double *d_f, const double *d_bc, int nz,
                                            int plane_stride, void *stream, sx_solve_stats *stats) {
  if (!s || !d_u || !d_f || plane_stride < s->mesh->nel * s->mesh->npnp) return SX_ERR_ARG;
  if (nz <= 0 || (nz > 1 && (nz % 2 || nz / 2 > s->num_modes))) return SX_ERR_ARG;
  // the factors and element matrices live on the mesh's device; the scratch
  // array is taken on the current one: they must be the same device
  SX_TRY(check_mesh_device(*s->mesh, "sx_field_solve_device_static"));
  const sx_mesh_s &Mh = *s->mesh;
  const int ngroups = nz == 1 ? 1 : nz / 2;
  // Scratch layout: [one Job][rhs: P * npad][Fb: P * nel * next][gess: P * nglobal],
  // reused by every mode in turn (the modes run one after another on `stream`).
  size_t need = 0;
  for (int l = 0; l < ngroups; l++) {
    const PlaneGroup g = plane_group(s->base_mode, nz, l);
    const System &S = *s->sys[g.mode];
    if (S.method != SX_DIRECT) {
      set_error("sx_field_solve_device_static: local mode %d is not a DIRECT system (JACPCG needs the "
                "allocating entry sx_field_solve_device)",
                g.mode);
      return SX_ERR_UNSUPPORTED;
    }
    const size_t npad = (size_t)std::max(S.nblk, 1) * NB;
    const size_t b = align256(sizeof(Job)) + align256((size_t)g.P * npad * 8) +
                     align256((size_t)g.P * Mh.nel * Mh.next * 8) + align256((size_t)g.P * Mh.nglobal * 8);
    need = std::max(need, b);
  }
  if (need > (size_t)SX_STATIC_SCRATCH_BYTES) {
    set_error("sx_field_solve_device_static: this solve needs %zu bytes of scratch per mode; the static "
              "scratch holds %zu (SX_STATIC_SCRATCH_BYTES)",
              need, (size_t)SX_STATIC_SCRATCH_BYTES);
    return SX_ERR_CAPACITY;
  }
  void *base = nullptr;
  SX_TRY(scratch_on_current_device(&base));
  unsigned char *sp = static_cast<unsigned char *>(base);
  Job *djob = reinterpret_cast<Job *>(sp);
  cudaStream_t st = (cudaStream_t)stream;
  const MeshView M = s->mesh->view();
  SX_TRY(prepare_direct_kernels(M));
  const BandSched sc = s->sched(1);
  const long long bcstride = (long long)std::max(Mh.nbound, 1) * Mh.np;
  // one host Job, reused: the 1-element vector is allocated once per thread
  // (direct_solve_jobs reads the host copy only while it enqueues)
  thread_local std::vector<Job> one(1);
  sx_solve_stats loc{};
  for (int l = 0; l < ngroups; l++) {
    const PlaneGroup g = plane_group(s->base_mode, nz, l);
    const System &S = *s->sys[g.mode];
    Job &j = one[0];
    std::memset(&j, 0, sizeof(j));
    j.u = d_u + (long long)g.plane0 * plane_stride;
    j.f = d_f + (long long)g.plane0 * plane_stride;
    j.bc = d_bc ? d_bc + (long long)g.plane0 * bcstride : nullptr;
    j.ustride = j.fstride = plane_stride;
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
    j.rhs_stride = j.npad;
    size_t off = align256(sizeof(Job));
    j.rhs = reinterpret_cast<double *>(sp + off);
    off += align256((size_t)g.P * j.npad * 8);
    j.Fb = reinterpret_cast<double *>(sp + off);
    off += align256((size_t)g.P * Mh.nel * Mh.next * 8);
    j.gess = reinterpret_cast<double *>(sp + off);
    j.pc = S.pc.p;
    j.status = s->dstatus.p;
    // Stream-ordered after the previous mode's kernels, which read the same
    // slot.  What must start at zero is gess (the essential values):
    // direct_solve_jobs clears it with cudaMemsetAsync before k_essential
    // writes the boundary values.  rhs (padding included) and Fb are written
    // in full by k_rhs_dss / k_rhs_elem before anything reads them.
    k_put_job<<<1, 32, 0, st>>>(djob, j);
    SX_CUDA(cudaGetLastError());
    int nl = 0;
    SX_TRY(direct_solve_jobs(M, djob, one, st, sc, &nl));
    loc.kernel_launches += nl + 1;
    loc.planes_solved += g.P;
  }
  SX_CUDA(cudaGetLastError());
  if (stats) *stats = loc;
  return SX_OK;
}
