/*
 * semtex_b200.h -- C ABI of the B200 per-Fourier-mode Helmholtz solver.
 *
 * Drop-in boundary for semtex's elliptic solve.  Each entry point names the
 * reference interface it replaces (file:line in the semtex tree).  All calls
 * return an int status (SX_OK == 0); nothing calls exit(), unlike
 * message(..., ERROR) in the reference (veclib/util.c:24-46).
 *
 * Data layout (same as the reference's AuxField planes, src/auxfield.cpp:31-54):
 *   a plane holds nel elements, each np*np values row-major
 *   (src/element.h:23-24); planes are `plane_stride` doubles apart
 *   (Geometry::planeSize, src/geometry.cpp:103-109); plane 0 is mode 0,
 *   plane 1 the Nyquist datum (skipped, as at src/field.cpp:566),
 *   planes 2k / 2k+1 the real / imaginary parts of mode k
 *   (femlib/fourier.c:63-69).
 *
 * Boundary-condition lines: for each plane, nbound*np values, boundary b's
 * np values at its side nodes in CCW order (the reference's Field::_line,
 * src/field.cpp:51-73).
 *
 * Threading: an sx_mesh / sx_modal may be used from one host thread at a
 * time.  Calls on different handles may run concurrently on different
 * streams.
 */
#ifndef SEMTEX_B200_H
#define SEMTEX_B200_H

#if defined(__GNUC__)
#define SX_API __attribute__((visibility("default")))
#else
#define SX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  SX_OK = 0,
  SX_ERR_ARG = 1,           /* invalid argument                                   */
  SX_ERR_CUDA = 2,          /* CUDA runtime error                                 */
  SX_ERR_NOMEM = 3,         /* device or host allocation failed                   */
  SX_ERR_JACOBIAN = 4,      /* nonpositive Jacobian (src/element.cpp:1349-1352)   */
  SX_ERR_SINGULAR_HII = 5,  /* singular interior block (src/element.cpp:212-216)  */
  SX_ERR_NOT_SPD = 6,       /* band factor failed (src/matrix.cpp:259-261)        */
  SX_ERR_BAND = 7,          /* btog couples nodes further apart than nband        */
  SX_WARN_STEP_LIMIT = 8,   /* PCG step limit reached (a warning in the
                               reference, src/field.cpp:706); solution returned  */
  SX_ERR_UNSUPPORTED = 9,   /* e.g. np outside [3, 12], cylindrical geometry       */
  SX_ERR_TIMEOUT = 10,      /* a bounded device-side wait ran out                 */
  SX_ERR_CAPACITY = 11,     /* serving: request larger than the memory budget     */
  SX_ERR_NOT_FOUND = 12     /* serving: unknown request id                        */
};

/* Solver kinds: femlib/cfemdef.h:43-47 (SolverKind).  SX_AUTO has no
 * reference counterpart: each mode is DIRECT when the band Cholesky streams
 * fewer bytes than Jacobi-PCG would for its conditioning (the routing rule
 * of SX_TUNE_MIXED_ROUTE), JACPCG otherwise. */
enum { SX_DIRECT = 0, SX_JACPCG = 1, SX_MIXED = 2, SX_AUTO = 3 };

/* Boundary-condition kinds (src/condition.h: Essential, Natural, Mixed). */
enum { SX_BC_ESSENTIAL = 0, SX_BC_NATURAL = 1, SX_BC_MIXED = 2 };

/* Precision of the batched form. */
enum { SX_FP64 = 0, SX_MIXED_FP32 = 1 };

typedef struct sx_mesh_s *sx_mesh;
typedef struct sx_modal_s *sx_modal;

/* Mesh description: what semtex's vector<Element*> + BoundarySys/NumberSys
 * carry into MatrixSys and Field::solve.  All arrays are host memory and are
 * copied; the caller keeps ownership. */
typedef struct {
  int np;               /* knots per element side, Geometry::nP()              */
  int nel;              /* elements, Geometry::nElmt()                          */
  const double *x;      /* nel*np*np node x, Element::_xmesh                    */
  const double *y;      /* nel*np*np node y, Element::_ymesh                    */
  const int *btog;      /* nel*4*(np-1), NumberSys::btog() (src/numbersys.h:59) */
  const int *bmask;     /* nel*4*(np-1), NumberSys::bmask()                     */
  int nglobal;          /* NumberSys::nGlobal()                                 */
  int nsolve;           /* NumberSys::nSolve()                                  */
  int nband;            /* NumberSys::nBand(), band incl. diagonal              */
  int nbound;           /* boundary edges (BoundarySys::nSurf())                */
  const int *b_elmt;    /* nbound: element of each boundary edge                */
  const int *b_side;    /* nbound: side 0..3 (CCW, side 0 at s = -1)            */
  const int *b_kind;    /* nbound: SX_BC_*                                      */
  const double *b_K;    /* nbound or NULL: Mixed K  (src/condition.cpp:247-262) */
  const double *b_C;    /* nbound or NULL: Mixed C                              */
} sx_mesh_desc;

/* Solve statistics. */
typedef struct {
  int planes_solved;    /* planes actually solved (Nyquist excluded)            */
  int iterations_max;   /* PCG: max iterations over planes (0 for DIRECT)       */
  int iterations_total; /* PCG: sum over planes                                 */
  int refinements;      /* mixed precision: outer refinement steps taken        */
  double final_rel_residual; /* mixed precision / PCG: max ||r||/||b||          */
  int kernel_launches;  /* kernels this call enqueued (graph nodes included)    */
  int planes_direct;    /* mixed precision: planes routed to the FP64 band solve */
} sx_solve_stats;

/* ---- library ------------------------------------------------------------ */
SX_API const char *sx_version(void);
SX_API const char *sx_status_string(int status);
/* Human-readable detail of the last failing call on this host thread. */
SX_API const char *sx_last_error(void);
/* Device used by subsequent calls from this host thread (cudaSetDevice). */
SX_API int sx_set_device(int device);
/* Limit of the bounded device-side waits on the current device (no
 * reference counterpart): the band sweeps' waits for tiles and for solved
 * blocks, and the FP32 iterations' wait for their staged copies.  A wait that
 * runs out records SX_ERR_TIMEOUT, which the entry point (or
 * sx_modal_status) returns; the kernel still returns normally and the
 * context stays usable.  ms < 0 restores the defaults (about 2 s for the
 * sweeps, 1 s for the iterations); ms = 0 makes every such wait give up at
 * its first unsuccessful probe (to exercise the error path). */
SX_API int sx_set_wait_limit(double ms);

/* ---- mesh: replaces Element construction + BCmgr numbering ---------------
 * Element::Element / Element::mapping (src/element.cpp:30-100, 1281-1436),
 * BCmgr::buildnum emask (src/bcmgr.cpp:797-803), Edge::Edge area factors
 * (src/edge.cpp:35-80).  Geometry factors are computed on the host in FP64
 * and kept resident on the device. */
SX_API int sx_mesh_create(const sx_mesh_desc *desc, sx_mesh *out);
SX_API int sx_mesh_destroy(sx_mesh mesh);
/* Read back element e's geometric factors Q1,Q2,Q3,Q4,Q8 (np*np each). */
SX_API int sx_mesh_geometry(sx_mesh mesh, int e, double *q1, double *q2, double *q3, double *q4,
                     double *q8);
/* Read back element e's inverse mapping partials dr/dx, dr/dy, ds/dx, ds/dy
 * (np*np each; zero where the null-mapping rule of src/element.cpp:1431-1434
 * drops them) and, when imass is not NULL, the inverse assembled boundary
 * mass (nglobal doubles, src/bcmgr.cpp:805-821).  Any pointer may be NULL. */
SX_API int sx_mesh_partials(sx_mesh mesh, int e, double *drdx, double *drdy, double *dsdx, double *dsdy,
                            double *imass);
/* The band factor's envelope in tiles of 64 x 64: *nblk block columns of
 * nsolve; when env is not NULL it receives 2 * nblk ints, env[k] the tiles
 * above the diagonal of block column k that can be non-zero and
 * env[nblk + k] those right of the diagonal in block row k.  Every other tile
 * of the band (nband wide, as LAPACK's dpbtrf stores it, src/matrix.cpp:
 * 236-262) is an exact zero of the factor; the factorisation and the sweeps
 * skip them.  No counterpart in the reference, which stores and sweeps the
 * whole band. */
SX_API int sx_mesh_envelope(sx_mesh mesh, int *nblk, int *env);
/* The same tables from a mesh description, on the host alone (no device is
 * touched): to size the factor's storage before a mesh is created.  Reads
 * np, nel, btog, nglobal, nsolve and nband of desc. */
SX_API int sx_mesh_desc_envelope(const sx_mesh_desc *desc, int *nblk, int *env);

/* ---- modal system: replaces ModalMatrixSys::ModalMatrixSys ---------------
 * src/matrix.cpp:33-110, MatrixSys::MatrixSys src/matrix.cpp:139-317.
 * For each mode k in [base_mode, base_mode+num_modes): betak2 = (beta k)^2
 * (src/field.cpp:1121-1139).  DIRECT builds per-element hbi*hii^-1, hii^-1
 * and the banded Cholesky factor on the GPU (FP64); JACPCG builds the
 * inverse diagonal; MIXED is DIRECT for mode 0 and JACPCG otherwise
 * (src/matrix.cpp:93-96).  Systems with equal (lambda2, betak2) are shared,
 * as the reference's MS cache shares them (src/matrix.cpp:85-102). */
SX_API int sx_modal_create(sx_mesh mesh, double lambda2, double beta, int base_mode, int num_modes,
                    int method, sx_modal *out);
/* Same, with an explicit (lambda2, betak2) per local mode. */
SX_API int sx_modal_create_ex(sx_mesh mesh, int base_mode, int num_modes, const double *lambda2,
                       const double *betak2, int method, sx_modal *out);
/* ModalMatrixSys::~ModalMatrixSys, src/matrix.cpp:113-130. */
SX_API int sx_modal_destroy(sx_modal modal);
/* Status of the device work enqueued so far on this system: synchronises
 * the device, returns SX_OK or the first recorded device-side error (e.g.
 * SX_ERR_TIMEOUT from a bounded wait) and clears it. */
SX_API int sx_modal_status(sx_modal modal);
/* Device memory held by the modal system (factors, element matrices). */
SX_API unsigned long long sx_modal_device_bytes(sx_modal modal);
/* Band factor of local mode m, in LAPACK "U" band storage
 * (ldab = nband, veclib/lapack.h:107-108): nsolve*nband doubles. */
SX_API int sx_modal_band(sx_modal modal, int m, double *ab, int *nsolve, int *singular);

/* ---- solve: replaces Field::solve (src/field.cpp:509-725) ----------------
 * Plain form: FP64, mode by mode, same semantics as the reference:
 *   u   nz planes: in = initial guess (used by JACPCG), out = solution
 *   f   nz planes: forcing, overwritten (as src/field.cpp:525-526)
 *   bc  nz * nbound * np boundary-line values (NULL = all zero)
 * tol_rel / step_max: TOL_REL / STEP_MAX for JACPCG (femlib/defaults.h:29,89).
 * Host pointers; the copies are part of the call.  Every solve entry point
 * returns SX_ERR_ARG when the calling thread's current device is not the
 * one the mesh was created on (its systems live there). */
SX_API int sx_field_solve(sx_modal modal, double *u, double *f, const double *bc, int nz,
                   int plane_stride, double tol_rel, int step_max, sx_solve_stats *stats);
/* Same on device pointers, enqueued on `stream` (a cudaStream_t, NULL =
 * legacy default stream). */
SX_API int sx_field_solve_device(sx_modal modal, double *d_u, double *d_f, const double *d_bc, int nz,
                          int plane_stride, double tol_rel, int step_max, void *stream,
                          sx_solve_stats *stats);

/* ---- no-allocation direct solve (no reference counterpart) ---------------
 * sx_field_solve_device on DIRECT systems, with its per-call scratch (job
 * record, condensed right-hand sides, element boundary forcing, essential
 * values) in one file-scope device array of SX_STATIC_SCRATCH_BYTES instead
 * of the modal system's grow-only workspace: no cudaMalloc, cudaFree or other
 * device allocation in any call.  For callers that cannot allocate: loops
 * whose device memory is already held by another allocator (cudaMalloc would
 * fail) and latency-bound loops (cudaFree synchronises the device).
 *   - The first call on each device looks up the array's address with
 *     cudaGetSymbolAddress (with that device current), which can load the
 *     module; make that first call before any stream capture.
 *   - SX_ERR_CAPACITY when one mode needs more than SX_STATIC_SCRATCH_BYTES
 *     (sx_last_error() gives the bytes needed); SX_ERR_UNSUPPORTED when a
 *     mode's system is not DIRECT; SX_ERR_ARG when the current device is not
 *     the mesh's (the array used is the current device's).
 *   - Each mode's job record is written into the array by a one-thread
 *     kernel that takes the record as its argument, so no host memory is
 *     read after the call returns.
 *   - The array is shared by all calls on a device: calls that overlap in
 *     time (two threads or two streams) race on it; serialise them.
 *   - Results equal sx_field_solve_device's bit for bit (same kernels). */
#define SX_STATIC_SCRATCH_BYTES (4u << 20)
SX_API int sx_field_solve_device_static(sx_modal modal, double *d_u, double *d_f, const double *d_bc, int nz,
                                        int plane_stride, void *stream, sx_solve_stats *stats);

/* ---- batched form (no reference counterpart: extends Field::solve) --------
 * All modes of the system in one captured CUDA graph, every mode's planes
 * processed together.  precision = SX_FP64 (same answer as the plain form
 * to rounding) or SX_MIXED_FP32 (FP32 operator / interior / inner PCG,
 * FP64 band Cholesky, residual and refinement update; stops when the FP64
 * relative residual is <= tol_rel). */
SX_API int sx_field_solve_batched(sx_modal modal, double *d_u, double *d_f, const double *d_bc, int nz,
                           int plane_stride, int precision, double tol_rel, int max_refine,
                           void *stream, sx_solve_stats *stats);
/* Batched form on HOST buffers: copies f (and bc) to the device, solves,
 * copies u back; synchronous.  u is output only (the solve starts from
 * zero).  Pinned (page-locked) host buffers give full copy bandwidth. */
SX_API int sx_field_solve_batched_host(sx_modal modal, double *u, const double *f, const double *bc,
                                int nz, int plane_stride, int precision, double tol_rel,
                                int max_refine, sx_solve_stats *stats);

/* Schedule knobs of the batched forms (no reference counterpart), set by
 * the autotuner or by hand; value <= 0 restores the default.
 *   SX_TUNE_INNER_ITERS   FP32 PCG iterations per refinement round, at
 *                         least (12); raised per call to what the
 *                         worst-conditioned FP32-routed mode needs
 *   SX_TUNE_BAND_CLUSTER  CTAs per cluster in the band sweeps (auto)
 *   SX_TUNE_MIXED_ROUTE   how SX_MIXED_FP32 solves each mode: 0 = by cost
 *                         (default: modes whose Jacobi-CG would stream more
 *                         bytes than three band solves go to the FP64 band
 *                         Cholesky, when the mode is factored), 1 = FP32 CG
 *                         for every mode, 2 = band Cholesky for every
 *                         factored mode
 *   SX_TUNE_BAND_STAGES   band-sweep tiles in flight per CTA, 1..4 (auto:
 *                         4, or 2 or 1 when that lets a larger cluster
 *                         stay resident -- two CTAs then share an SM)
 *   SX_TUNE_BAND_LEAD     the cluster leader's share of the band tiles off
 *                         the critical path: K in 2..64 gives it the last of
 *                         every K such tiles of a block column (worked on
 *                         while it waits for the other CTAs' partial sums);
 *                         1 = none (it keeps only the tile next to the
 *                         diagonal and the diagonal block's inverse);
 *                         <= 0 = the default
 *   SX_TUNE_HOST_CHUNK    Fourier modes per chunk of the host-buffer
 *                         pipeline of sx_field_solve_batched_host (each
 *                         chunk is copied up, solved and copied back on
 *                         its own streams, overlapping the others); auto:
 *                         eight chunks of at least 8 modes when every mode
 *                         goes to the band Cholesky and there are 32 or
 *                         more, else half the modes rounded up to a
 *                         multiple of 16                                   */
enum {
  SX_TUNE_INNER_ITERS = 1,
  SX_TUNE_BAND_CLUSTER = 2,
  SX_TUNE_MIXED_ROUTE = 3,
  SX_TUNE_BAND_STAGES = 4,
  SX_TUNE_BAND_LEAD = 5,
  SX_TUNE_HOST_CHUNK = 6
};
SX_API int sx_modal_tune(sx_modal modal, int knob, int value);

/* Autotuner (no reference counterpart): times the batched form on the
 * caller's own data for each candidate schedule and keeps the fastest in the
 * modal system for launches over that many systems (the band-sweep knobs
 * set by hand give way to it; launches over other numbers of systems, e.g.
 * the chunks of the host-buffer entry, keep their default) --
 *   the band-sweep cluster size (CTAs sharing one system's tiles; sizes the
 *   SM groups cannot hold are skipped) and ring depth (4, 2 or 1 tiles in
 *   flight per CTA), then the leader's share of the tiles on the best of
 *   them, for SX_FP64 and for the modes that SX_MIXED_FP32 routes to the
 *   band Cholesky;
 *   the floor on FP32 iterations per refinement round, for SX_MIXED_FP32.
 * d_f is only read (each trial solves a copy, allocated for the duration);
 * d_u holds the last trial's solution.  Candidates whose solve does not
 * reach tol_rel are kept only when none does. */
typedef struct {
  int band_cluster; /* chosen CTAs per cluster (0: the form runs no band sweeps) */
  int inner_iters;  /* chosen floor on FP32 iterations per round (0: FP64 form) */
  double ms;        /* one solve with the chosen schedule                     */
  int trials;       /* schedules timed                                        */
  int band_stages;  /* chosen band-sweep ring depth (0: no band sweeps)       */
  int band_lead;    /* chosen leader share K (0: none, as knob value 1)       */
} sx_tune_result;
SX_API int sx_modal_autotune(sx_modal modal, double *d_u, const double *d_f, const double *d_bc, int nz,
                             int plane_stride, int precision, double tol_rel, int max_refine, void *stream,
                             sx_tune_result *out);

/* Profiling hook (no reference counterpart): re-launch only the banded
 * forward/backward sweeps of the last batched solve `reps` times on
 * `stream`, so the dominant kernel can be timed on its own.  The RHS
 * workspace is overwritten; call after sx_field_solve_batched. */
SX_API int sx_profile_band_sweeps(sx_modal modal, int reps, void *stream);
/* Same for the mixed-precision form: `reps` launches of one inner FP32
 * iteration (the fused k_cg kernel) on the workspace of the last mixed
 * solve (which needs >= 2 inner iterations).  The iterates are overwritten;
 * the next solve starts afresh. */
SX_API int sx_profile_mixed_iterations(sx_modal modal, int reps, void *stream);

/* ---- z-direction transform: replaces dDFTr as AuxField::transform uses it --
 * femlib/fourier.c:47-171, src/auxfield.cpp:1133-1170.  In place on device
 * data: nz planes plane_stride doubles apart, the first npts points of each
 * plane transformed along z.  sign = +1: physical -> Fourier, scaled by 1/nz,
 * planes ordered mode 0, Nyquist (real), then Re/Im of modes 1 .. nz/2 - 1
 * (the layout every solve entry point takes); sign = -1: back, unscaled.
 * nz = 1 is a no-op; otherwise nz must be even with prime factors 2, 3, 5.
 * Enqueued on `stream`; nz = 2, 4, ..., 64 run as one kernel and return at
 * once, other lengths (which share a workspace) are waited for. */
SX_API int sx_transform_z(double *d_data, int nz, int plane_stride, int npts, int sign, void *stream);

/* ---- DNS elliptic phase: the field operations around the Helmholtz solves --
 * Device data in the solve entry points' layout: nz planes plane_stride
 * doubles apart (the buffers hold nz * plane_stride doubles), each plane
 * nel*np*np points, element-major, np x np row-major.  Fourier planes are
 * ordered as the solves take them: with base_mode 0, plane 0 is mode 0 and
 * plane 1 Nyquist; planes 2k, 2k+1 hold Re, Im of mode k + base_mode.  Each
 * call is enqueued on `stream` and returns at once.  Padding beyond a
 * plane's points is neither read nor written (d/dz and the wave step aside,
 * which the reference also applies to it).  Cylindrical geometry (the
 * reference's mulY steps) is not supported by this library's meshes.
 *
 * AuxField::gradient (src/auxfield.cpp:514-616) in place: dir 0 d/dx, 1
 * d/dy (Element::grad, src/element.cpp:552-596, every plane); dir 2 d/dz of
 * Fourier planes (nz even): Re' = -beta k Im, Im' = beta k Re, the planes
 * of mode 0 and Nyquist zeroed when base_mode is 0. */
SX_API int sx_field_gradient(sx_mesh mesh, double *d_data, int nz, int plane_stride, int dir, double beta,
                             int base_mode, void *stream);
/* setPForce (dns/integrate.cpp:262-277): d_out = (sum_i d/dx_i us[i]) / dt
 * over ndim (2 or 3) components, summed x + y, then + z, then times 1/dt.
 * ndim 3 needs nz even; d_out may be us[0] or us[1], not us[2].  dt = 0 is
 * SX_ERR_ARG (the reference's "divide by zero"). */
SX_API int sx_dns_pressure_forcing(sx_mesh mesh, const double *const *d_us, int ndim, double *d_out, int nz,
                                   int plane_stride, double dt, double beta, int base_mode, void *stream);
/* project (dns/integrate.cpp:280-310): for the nadv advected fields,
 *   uf[i] = alpha us[i] (times prandtl for the scalar, index ncom, when
 *           nadv = ncom + 1) + (1/kinvis) d/dx_i p   for i < ndim,
 * alpha = -1/(dt kinvis); ncom velocity components, ndim <= ncom <= 3.
 * uf[i] may be us[i] (in place); no uf[i] may be p. */
SX_API int sx_dns_project(sx_mesh mesh, const double *const *d_us, const double *d_p, double *const *d_uf,
                          int ndim, int ncom, int nadv, int nz, int plane_stride, double dt, double kinvis,
                          double prandtl, double beta, int base_mode, void *stream);
/* Field::smooth (src/field.cpp:190-276) in place on every plane: the Q4-
 * weighted sum of each global node's element-boundary values, taken element
 * after element as bndryDsSum does (src/element.cpp:464-487), times the
 * inverse assembled mass, written back to every slot of the node
 * (bndryInsert).  Interior points are unchanged. */
SX_API int sx_field_smooth(sx_mesh mesh, double *d_data, int nz, int plane_stride, void *stream);
/* waveProp (dns/integrate.cpp:227-259): for each of nadv fields,
 *   h[i] = sum_{q < order} (-alpha_{q+1} us[q][i] + dt beta_q uf[q][i]),
 * alpha the stiffly-stable and beta the extrapolation weights of the given
 * order (1-3, src/integration.cpp:98-163), accumulated level by level as the
 * reference's axpy sequence does.  us, uf: order*nadv device pointers,
 * level-major (us[q*nadv + i] = level q of field i), npts doubles each; h[i]
 * may be any of its field's inputs. */
SX_API int sx_dns_wave_prop(const double *const *d_us, const double *const *d_uf, double *const *d_h, int nadv,
                            int order, long long npts, double dt, void *stream);

/* ---- field files: replace the Header writer and AuxField stream I/O -------
 * The reference's field-file format: a 10-line ASCII header (Header <<,
 * src/data2df.cpp:503-535; read by strm>>Domain, src/domain.cpp:284-400, and
 * by compare, utility/compare.cpp:112-175) and the fields' planes in binary,
 * field after field, plane after plane, nel*np*np doubles each
 * (ostream<<AuxField / istream>>AuxField, src/auxfield.cpp:997-1095).  Host
 * memory, planes plane_stride doubles apart (the padding of a plane read is
 * zeroed).  A file written on a machine of the other byte order is swapped
 * on reading (Domain's reader does the same). */
typedef struct {
  char session[256];  /* session name                                            */
  int np, nz, nel;    /* knots per element side, planes, elements                */
  int step;           /* time step number                                        */
  double time, dt, kinvis, beta;
  char fields[64];    /* one character per field, in file order, e.g. "uvwp"     */
  int swapped;        /* set by the readers: the file's byte order is not ours   */
} sx_field_header;
/* Write len(h->fields) fields, fields[f] = nz planes. */
SX_API int sx_field_write(const char *path, const sx_field_header *h, const double *const *fields,
                          int plane_stride);
SX_API int sx_field_read_header(const char *path, sx_field_header *h);
/* Read every field of the file into fields[f] (NULL skips field f). */
SX_API int sx_field_read(const char *path, sx_field_header *h, double *const *fields, int plane_stride);
/* compare-style norms of exact - computed on the GPU (device pointers, nz
 * planes of `mesh`): norms[2z] = max |exact - computed| over plane z (compare's
 * norm_inf, utility/compare.cpp:206-218), norms[2z+1] = AuxField::errors' L2
 * figure (src/auxfield.cpp:813-860: the elements' sqrt(sum e^2 Q4) summed,
 * over the summed element areas) at the fields' own GLL points.  norms is
 * host memory; the call waits for the result. */
SX_API int sx_field_norms(sx_mesh mesh, const double *d_computed, const double *d_exact, int nz,
                          int plane_stride, double *norms, void *stream);

/* ---- numbering files: replace BCmgr::buildnum's reader and enumerate's writer
 * The text file session.num (written by enumerate, printup in
 * utility/enumerate.cpp:426-537; read by BCmgr::buildnum, src/bcmgr.cpp:586-
 * 790): per number set NEL, NP_MAX, NEXT_MAX, NINT_MAX, NTOTAL, NBOUNDARY,
 * NGLOBAL, NSOLVE, OPTIMIZATION, BANDWIDTH (diagonal included), then per
 * element boundary slot (element, side, offset) the bmap (btog) and mask of
 * each set -- the same layout as sx_mesh_desc's btog and bmask.
 * sx_numbering_read takes the set whose name holds `field` (e.g. 'u' from set
 * "uv"), checks NEL, NP_MAX and NBOUNDARY against nel and np as the reader
 * does (SX_ERR_ARG on a mismatch), fills btog and bmask (nel*4*(np-1) each)
 * and returns NGLOBAL, NSOLVE, BANDWIDTH and the set's name (set_fields may be
 * NULL). */
SX_API int sx_numbering_read(const char *path, char field, int nel, int np, int *btog, int *bmask, int *nglobal,
                             int *nsolve, int *nband, char *set_fields, int set_fields_cap);
/* Write nset number sets in enumerate's layout (btog[j], bmask[j] of set j). */
SX_API int sx_numbering_write(const char *path, const char *fields, int nset, const char *const *set_fields,
                              int nel, int np, const int *const *btog, const int *const *bmask,
                              const int *nglobal, const int *nsolve, const int *nband, int optimization);

/* ---- multi-mesh batch (no reference counterpart) --------------------------
 * Solves the planes of several modal systems -- different meshes, element
 * counts, orders and mode sets -- together, on device buffers.  Each is the
 * batched form of that system (same answer as sx_field_solve_batched within
 * the stated tolerance), but the kernels cover all of them at once:
 *   SX_MIXED_FP32  one launch per kernel and element order covers the tiles
 *                  of every member of that order (the orders run side by
 *                  side); refinement rounds continue until every plane of
 *                  every member meets tol_rel;
 *   SX_FP64 (and the modes SX_MIXED_FP32 routes to the band Cholesky)
 *                  one band-sweep launch covers every member's systems.
 * The launch sequence is captured as CUDA graphs and replayed while the set
 * of members and their buffers stay the same.  A modal system may appear
 * once per call.  stats, when non-null, has `count` entries.  The batch
 * object holds the tables and graphs; it does not own the modal systems. */
typedef struct sx_batch_s *sx_batch;
SX_API int sx_batch_create(sx_batch *out);
SX_API int sx_batch_solve(sx_batch batch, int count, const sx_modal *modals, double *const *d_u,
                          double *const *d_f, const double *const *d_bc, const int *nz, const int *plane_stride,
                          int precision, double tol_rel, int max_refine, void *stream, sx_solve_stats *stats);
SX_API int sx_batch_destroy(sx_batch batch);

/* ---- serving loop (no reference counterpart) -----------------------------
 * A request loop for Helmholtz solves of different meshes, orders and mode
 * counts.  Requests are admitted in arrival order as device slots and memory
 * free up (bounded by hbm_budget).  Each slot takes every admissible pending
 * request (up to max_batch) and solves them together as one multi-mesh
 * batch (sx_batch_solve) on its own stream; the slots' batches run
 * concurrently, and requests that arrive meanwhile join the next batch.
 * Element geometry and per-mode systems (Jacobi diagonals, or factored
 * condensed matrices) stay resident across requests, keyed by (mesh,
 * lambda2, betak2, kind), with least-recently-used eviction.  A request's
 * result is the same alone or in a mix within the solve tolerance (the
 * FP64 form: to rounding). */
typedef struct sx_server_s *sx_server;

typedef struct {
  unsigned long long hbm_budget; /* device bytes for caches + in-flight work; 0 = 70% of free */
  int slots;                     /* requests on the device at once; 0 = 8                      */
  int precision;                 /* SX_MIXED_FP32 (PCG) or SX_FP64 (DIRECT, cached factors)     */
  double tol_rel;                /* mixed: FP64 relative residual target; 0 = 1e-12            */
  int max_refine;                /* mixed: refinement rounds cap; 0 = 30                        */
  int inner_iters;               /* mixed: FP32 PCG iterations per round; 0 = 12                */
  int max_batch;                 /* requests solved together by one slot; 0 = 8                 */
} sx_server_config;

typedef struct {
  const sx_mesh_desc *mesh;      /* copied at submit                                          */
  int base_mode, num_modes;
  const double *lambda2;         /* num_modes, copied                                         */
  const double *betak2;          /* num_modes, copied                                         */
  int nz, plane_stride;          /* planes in semtex order, as sx_field_solve                 */
  const double *f;               /* nz*plane_stride forcing, copied at submit                 */
  const double *bc;              /* nz*nbound*np or NULL, copied                              */
  double *u;                     /* nz*plane_stride, written before the request completes     */
} sx_request;

typedef struct {
  unsigned long long submitted, completed, failed, rejected;
  unsigned long long mesh_hits, mesh_misses, system_hits, system_misses, evictions;
  unsigned long long bytes_cached, bytes_budget;
  double p50_ms, p99_ms, mean_ms; /* submit-to-completion latency of completed requests     */
  unsigned long long batches;     /* batches served                                          */
  double queue_ms, build_ms, solve_ms; /* summed over requests: waiting for admission; geometry,
                                          system builds and factorisation; the batch solve with
                                          its host <-> device copies                            */
} sx_server_stats;

SX_API int sx_server_create(const sx_server_config *cfg, sx_server *out);
/* Queue a request; returns at once with its id.  SX_ERR_CAPACITY when the
 * request alone cannot fit in hbm_budget. */
SX_API int sx_server_submit(sx_server s, const sx_request *req, unsigned long long *id);
/* Wait for a request (timeout_s < 0: no limit); *status is its solve status. */
SX_API int sx_server_wait(sx_server s, unsigned long long id, double timeout_s, int *status,
                          double *latency_ms);
SX_API int sx_server_get_stats(sx_server s, sx_server_stats *st);
/* Finishes the queued requests, then releases everything. */
SX_API int sx_server_destroy(sx_server s);

#ifdef __cplusplus
}
#endif
#endif /* SEMTEX_B200_H */
