"""semtex_b200: B200-native per-Fourier-mode Helmholtz solves for semtex.

Python front-end over the C ABI in include/semtex_b200.h.  The classes mirror
the reference's solve interface:

* ``Mesh``            Elements + BoundarySys/NumberSys (src/element.h,
                      src/bsys.h, src/numbersys.h) resident on the GPU;
* ``ModalMatrixSys``  ModalMatrixSys (src/matrix.h:56-71): one MatrixSys per
                      Fourier mode, factored on the GPU;
* ``ModalMatrixSys.solve``  Field::solve (src/field.cpp:509-725): forcing is
                      overwritten, the solution returned.

The compute path is the compiled CUDA library; there is no CPU fallback.
If ``libsemtex_b200.so`` is missing, import fails; the library is mapped on
the first call into it (so that the mesh and workload builders can be used
without it, e.g. by a CPU-only timing of the oracle), and a library that
cannot be loaded fails that call.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .mesh import (ESSENTIAL, MIXED, NATURAL, Boundary, QuadMesh, gll_points,  # noqa: F401
                   rect_mesh)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsemtex_b200.so")

DIRECT, JACPCG, MIXED_SOLVER, AUTO = 0, 1, 2, 3
FP64, MIXED_FP32 = 0, 1
OK, WARN_STEP_LIMIT = 0, 8
TUNE_INNER_ITERS, TUNE_BAND_CLUSTER, TUNE_MIXED_ROUTE, TUNE_BAND_STAGES, TUNE_BAND_LEAD = 1, 2, 3, 4, 5
TUNE_HOST_CHUNK = 6
ROUTE_AUTO, ROUTE_CG, ROUTE_BAND = 0, 1, 2
STATIC_SCRATCH_BYTES = 4 << 20  # SX_STATIC_SCRATCH_BYTES


class SolverError(RuntimeError):
    def __init__(self, status, what):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} ({status}): {last_error()}")


class MeshDesc(C.Structure):
    _fields_ = [("np", C.c_int), ("nel", C.c_int),
                ("x", C.POINTER(C.c_double)), ("y", C.POINTER(C.c_double)),
                ("btog", C.POINTER(C.c_int)), ("bmask", C.POINTER(C.c_int)),
                ("nglobal", C.c_int), ("nsolve", C.c_int), ("nband", C.c_int),
                ("nbound", C.c_int),
                ("b_elmt", C.POINTER(C.c_int)), ("b_side", C.POINTER(C.c_int)),
                ("b_kind", C.POINTER(C.c_int)),
                ("b_K", C.POINTER(C.c_double)), ("b_C", C.POINTER(C.c_double))]


class SolveStats(C.Structure):
    _fields_ = [("planes_solved", C.c_int), ("iterations_max", C.c_int),
                ("iterations_total", C.c_int), ("refinements", C.c_int),
                ("final_rel_residual", C.c_double), ("kernel_launches", C.c_int),
                ("planes_direct", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneResult(C.Structure):
    _fields_ = [("band_cluster", C.c_int), ("inner_iters", C.c_int), ("ms", C.c_double),
                ("trials", C.c_int), ("band_stages", C.c_int), ("band_lead", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget", C.c_ulonglong), ("slots", C.c_int), ("precision", C.c_int),
                ("tol_rel", C.c_double), ("max_refine", C.c_int), ("inner_iters", C.c_int),
                ("max_batch", C.c_int)]


class Request(C.Structure):
    _fields_ = [("mesh", C.POINTER(MeshDesc)), ("base_mode", C.c_int), ("num_modes", C.c_int),
                ("lambda2", C.POINTER(C.c_double)), ("betak2", C.POINTER(C.c_double)),
                ("nz", C.c_int), ("plane_stride", C.c_int),
                ("f", C.POINTER(C.c_double)), ("bc", C.POINTER(C.c_double)),
                ("u", C.POINTER(C.c_double))]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_ulonglong) for n in
                ("submitted", "completed", "failed", "rejected", "mesh_hits", "mesh_misses",
                 "system_hits", "system_misses", "evictions", "bytes_cached", "bytes_budget")] + \
               [("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double),
                ("batches", C.c_ulonglong), ("queue_ms", C.c_double), ("build_ms", C.c_double),
                ("solve_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `python -m semtex_b200.build` "
                      "(no CPU fallback exists)")


class FieldHeader(C.Structure):
    _fields_ = [("session", C.c_char * 256), ("np", C.c_int), ("nz", C.c_int), ("nel", C.c_int),
                ("step", C.c_int), ("time", C.c_double), ("dt", C.c_double), ("kinvis", C.c_double),
                ("beta", C.c_double), ("fields", C.c_char * 64), ("swapped", C.c_int)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["session"] = self.session.decode()
        d["fields"] = self.fields.decode()
        return d


def _load():
    L = C.CDLL(LIB_PATH)
    vp, ip, dp = C.c_void_p, C.c_int, C.c_double
    P = C.POINTER
    L.sx_version.restype = C.c_char_p
    L.sx_status_string.restype = C.c_char_p
    L.sx_status_string.argtypes = [ip]
    L.sx_last_error.restype = C.c_char_p
    L.sx_set_device.argtypes = [ip]
    L.sx_set_wait_limit.argtypes = [dp]
    L.sx_mesh_create.argtypes = [P(MeshDesc), P(vp)]
    L.sx_mesh_destroy.argtypes = [vp]
    L.sx_mesh_geometry.argtypes = [vp, ip] + [P(dp)] * 5
    L.sx_modal_create.argtypes = [vp, dp, dp, ip, ip, ip, P(vp)]
    L.sx_modal_create_ex.argtypes = [vp, ip, ip, P(dp), P(dp), ip, P(vp)]
    L.sx_modal_destroy.argtypes = [vp]
    L.sx_modal_device_bytes.argtypes = [vp]
    L.sx_modal_device_bytes.restype = C.c_ulonglong
    L.sx_modal_band.argtypes = [vp, ip, P(dp), P(ip), P(ip)]
    L.sx_field_solve.argtypes = [vp, P(dp), P(dp), P(dp), ip, ip, dp, ip, P(SolveStats)]
    L.sx_field_solve_device.argtypes = [vp, vp, vp, vp, ip, ip, dp, ip, vp, P(SolveStats)]
    L.sx_field_solve_device_static.argtypes = [vp, vp, vp, vp, ip, ip, vp, P(SolveStats)]
    L.sx_field_solve_batched.argtypes = [vp, vp, vp, vp, ip, ip, ip, dp, ip, vp, P(SolveStats)]
    L.sx_field_solve_batched_host.argtypes = [vp, P(dp), P(dp), P(dp), ip, ip, ip, dp, ip,
                                              P(SolveStats)]
    L.sx_profile_band_sweeps.argtypes = [vp, ip, vp]
    L.sx_profile_mixed_iterations.argtypes = [vp, ip, vp]
    L.sx_modal_status.argtypes = [vp]
    L.sx_modal_tune.argtypes = [vp, ip, ip]
    L.sx_modal_autotune.argtypes = [vp, vp, vp, vp, ip, ip, ip, dp, ip, vp, P(TuneResult)]
    L.sx_transform_z.argtypes = [vp, ip, ip, ip, ip, vp]
    L.sx_mesh_partials.argtypes = [vp, ip] + [P(dp)] * 5
    L.sx_mesh_envelope.argtypes = [vp, P(ip), P(ip)]
    L.sx_mesh_desc_envelope.argtypes = [P(MeshDesc), P(ip), P(ip)]
    L.sx_field_gradient.argtypes = [vp, vp, ip, ip, ip, dp, ip, vp]
    L.sx_dns_pressure_forcing.argtypes = [vp, P(vp), ip, vp, ip, ip, dp, dp, ip, vp]
    L.sx_dns_project.argtypes = [vp, P(vp), vp, P(vp), ip, ip, ip, ip, ip, dp, dp, dp, dp, ip, vp]
    L.sx_field_smooth.argtypes = [vp, vp, ip, ip, vp]
    L.sx_dns_wave_prop.argtypes = [P(vp), P(vp), P(vp), ip, ip, C.c_longlong, dp, vp]
    L.sx_field_write.argtypes = [C.c_char_p, P(FieldHeader), P(P(dp)), ip]
    L.sx_field_read_header.argtypes = [C.c_char_p, P(FieldHeader)]
    L.sx_field_read.argtypes = [C.c_char_p, P(FieldHeader), P(P(dp)), ip]
    L.sx_field_norms.argtypes = [vp, vp, vp, ip, ip, P(dp), vp]
    L.sx_numbering_read.argtypes = [C.c_char_p, C.c_char, ip, ip, P(ip), P(ip), P(ip), P(ip), P(ip),
                                    C.c_char_p, ip]
    L.sx_numbering_write.argtypes = [C.c_char_p, C.c_char_p, ip, P(C.c_char_p), ip, ip, P(P(ip)), P(P(ip)),
                                     P(ip), P(ip), P(ip), ip]
    L.sx_batch_create.argtypes = [P(vp)]
    L.sx_batch_destroy.argtypes = [vp]
    L.sx_batch_solve.argtypes = [vp, ip, P(vp), P(vp), P(vp), P(vp), P(ip), P(ip), ip, dp, ip, vp,
                                 P(SolveStats)]
    L.sx_server_create.argtypes = [P(ServerConfig), P(vp)]
    L.sx_server_submit.argtypes = [vp, P(Request), P(C.c_ulonglong)]
    L.sx_server_wait.argtypes = [vp, C.c_ulonglong, dp, P(ip), P(dp)]
    L.sx_server_get_stats.argtypes = [vp, P(ServerStats)]
    L.sx_server_destroy.argtypes = [vp]
    return L


class _Library:
    """The C ABI, mapped on first use (``lib.sx_*``)."""

    _handle = None

    def __getattr__(self, name):
        if _Library._handle is None:
            _Library._handle = _load()
        return getattr(_Library._handle, name)

    @property
    def loaded(self):
        return _Library._handle is not None


lib = _Library()


def status_string(s):
    return lib.sx_status_string(s).decode()


def last_error():
    return lib.sx_last_error().decode()


def version():
    return lib.sx_version().decode()


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _check(st, what, allow=(OK,)):
    if st not in allow:
        raise SolverError(st, what)
    return st


def mesh_desc(qm: QuadMesh):
    """sx_mesh_desc for a QuadMesh; returns (desc, arrays to keep alive)."""
    nb, be, bs, bk, bK, bC = qm.bc_arrays()
    k = dict(
        x=np.ascontiguousarray(qm.x, dtype=np.float64).reshape(-1),
        y=np.ascontiguousarray(qm.y, dtype=np.float64).reshape(-1),
        btog=np.ascontiguousarray(qm.btog, dtype=np.int32).reshape(-1),
        bmask=np.ascontiguousarray(qm.bmask, dtype=np.int32).reshape(-1),
        be=be.astype(np.int32), bs=bs.astype(np.int32), bk=bk.astype(np.int32),
        bK=bK.astype(np.float64), bC=bC.astype(np.float64))
    d = MeshDesc(qm.np, qm.nel, _dptr(k["x"]), _dptr(k["y"]), _iptr(k["btog"]),
                 _iptr(k["bmask"]), qm.nglobal, qm.nsolve, qm.nband, nb,
                 _iptr(k["be"]), _iptr(k["bs"]), _iptr(k["bk"]), _dptr(k["bK"]), _dptr(k["bC"]))
    return d, k


def band_envelope(qm: QuadMesh):
    """The band factor's envelope of a mesh by 64 x 64 tiles, computed on the
    host from its numbering alone (no device): (above, right), the tiles
    above the diagonal of each block column and right of it in each block
    row that the factorisation and the sweeps visit."""
    d, keep = mesh_desc(qm)
    nb = C.c_int()
    _check(lib.sx_mesh_desc_envelope(C.byref(d), C.byref(nb), None), "sx_mesh_desc_envelope")
    env = np.zeros(2 * max(nb.value, 1), dtype=np.int32)
    _check(lib.sx_mesh_desc_envelope(C.byref(d), C.byref(nb), env.ctypes.data_as(C.POINTER(C.c_int))),
           "sx_mesh_desc_envelope")
    del keep
    return env[:nb.value].copy(), env[nb.value:2 * nb.value].copy()


class Mesh:
    """A QuadMesh uploaded to the GPU (geometry factors + numbering)."""

    def __init__(self, qm: QuadMesh):
        self.qm = qm
        d, self._keep = mesh_desc(qm)
        h = C.c_void_p()
        _check(lib.sx_mesh_create(C.byref(d), C.byref(h)), "sx_mesh_create")
        self.h = h

    def partials(self, e):
        """Element e's (drdx, drdy, dsdx, dsdy) and the inverse boundary
        mass (nglobal)."""
        out = [np.zeros(self.qm.npnp) for _ in range(4)] + [np.zeros(self.qm.nglobal)]
        _check(lib.sx_mesh_partials(self.h, e, *[_dptr(a) for a in out]), "sx_mesh_partials")
        return out

    def envelope(self):
        """The band factor's envelope by 64 x 64 tiles: (above, right), the
        tiles above the diagonal of each block column and right of it in
        each block row that the factorisation and the sweeps visit."""
        nb = C.c_int()
        _check(lib.sx_mesh_envelope(self.h, C.byref(nb), None), "sx_mesh_envelope")
        env = np.zeros(2 * max(nb.value, 1), dtype=np.int32)
        _check(lib.sx_mesh_envelope(self.h, C.byref(nb), env.ctypes.data_as(C.POINTER(C.c_int))),
               "sx_mesh_envelope")
        return env[:nb.value].copy(), env[nb.value:2 * nb.value].copy()

    def geometry(self, e):
        out = [np.zeros(self.qm.npnp) for _ in range(5)]
        _check(lib.sx_mesh_geometry(self.h, e, *[_dptr(a) for a in out]), "sx_mesh_geometry")
        return out

    def close(self):
        if getattr(self, "h", None) and lib is not None:
            lib.sx_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class ModalMatrixSys:
    """One Helmholtz system per Fourier mode (ModalMatrixSys, src/matrix.cpp:33-110).

    Either ``lambda2`` (scalar) with ``beta`` (betak2 = (beta k)^2), or
    per-mode arrays ``lambda2_modes`` / ``betak2_modes``.
    """

    def __init__(self, mesh: Mesh, lambda2=0.0, beta=0.0, base_mode=0, num_modes=1,
                 method=DIRECT, lambda2_modes=None, betak2_modes=None):
        self.mesh = mesh
        self.base_mode, self.num_modes, self.method = base_mode, num_modes, method
        h = C.c_void_p()
        if lambda2_modes is None:
            _check(lib.sx_modal_create(mesh.h, float(lambda2), float(beta), base_mode, num_modes,
                                       method, C.byref(h)), "sx_modal_create")
        else:
            lam = np.ascontiguousarray(lambda2_modes, dtype=np.float64)
            bk2 = (np.zeros(num_modes) if betak2_modes is None
                   else np.ascontiguousarray(betak2_modes, dtype=np.float64))
            _check(lib.sx_modal_create_ex(mesh.h, base_mode, num_modes, _dptr(lam), _dptr(bk2),
                                          method, C.byref(h)), "sx_modal_create_ex")
        self.h = h

    @property
    def device_bytes(self):
        return int(lib.sx_modal_device_bytes(self.h))

    def band(self, m=0):
        """Factored band of local mode m in LAPACK "U" storage (nsolve, nband)."""
        ns, sg = C.c_int(), C.c_int()
        _check(lib.sx_modal_band(self.h, m, None, C.byref(ns), C.byref(sg)), "sx_modal_band")
        ab = np.zeros(ns.value * self.mesh.qm.nband)
        _check(lib.sx_modal_band(self.h, m, _dptr(ab), C.byref(ns), C.byref(sg)), "sx_modal_band")
        return ab.reshape(ns.value, self.mesh.qm.nband), bool(sg.value)

    def _bc_array(self, bc, nz):
        qm = self.mesh.qm
        nb = max(len(qm.boundaries), 1)
        if bc is None:
            return None
        return np.ascontiguousarray(np.broadcast_to(bc, (nz, nb, qm.np)), dtype=np.float64).copy()

    def solve(self, forcing, bc=None, u0=None, tol_rel=1e-8, step_max=500, return_stats=False):
        """Field::solve on host arrays.  forcing: (nz, nplane); returns u."""
        qm = self.mesh.qm
        f = np.ascontiguousarray(forcing, dtype=np.float64).reshape(-1, qm.nplane).copy()
        nz = f.shape[0]
        u = (np.zeros_like(f) if u0 is None
             else np.ascontiguousarray(u0, dtype=np.float64).reshape(nz, qm.nplane).copy())
        b = self._bc_array(bc, nz)
        st = SolveStats()
        rc = lib.sx_field_solve(self.h, _dptr(u), _dptr(f), _dptr(b) if b is not None else None,
                                nz, qm.nplane, tol_rel, step_max, C.byref(st))
        _check(rc, "sx_field_solve", allow=(OK, WARN_STEP_LIMIT))
        return (u, st.as_dict()) if return_stats else u

    def solve_device(self, d_u, d_f, d_bc, nz, stride, tol_rel=1e-8, step_max=500, stream=0):
        """Field::solve on device pointers (ints), enqueued on `stream`."""
        st = SolveStats()
        rc = lib.sx_field_solve_device(self.h, d_u, d_f, d_bc, nz, stride, tol_rel, step_max,
                                       stream, C.byref(st))
        _check(rc, "sx_field_solve_device", allow=(OK, WARN_STEP_LIMIT))
        return st.as_dict()

    def solve_device_static(self, d_u, d_f, d_bc, nz, stride, stream=0):
        """solve_device for DIRECT systems with no device allocation: scratch
        is a fixed device array of STATIC_SCRATCH_BYTES shared by all calls
        on a device (overlapping calls race; serialise them)."""
        st = SolveStats()
        rc = lib.sx_field_solve_device_static(self.h, d_u, d_f, d_bc, nz, stride, stream, C.byref(st))
        _check(rc, "sx_field_solve_device_static")
        return st.as_dict()

    def solve_batched(self, d_u, d_f, d_bc, nz, stride, precision=FP64, tol_rel=1e-12,
                      max_refine=8, stream=0):
        """All modes in one captured graph (device pointers)."""
        st = SolveStats()
        rc = lib.sx_field_solve_batched(self.h, d_u, d_f, d_bc, nz, stride, precision, tol_rel,
                                        max_refine, stream, C.byref(st))
        _check(rc, "sx_field_solve_batched", allow=(OK, WARN_STEP_LIMIT))
        return st.as_dict()

    def solve_batched_host(self, forcing, bc=None, out=None, precision=FP64, tol_rel=1e-12,
                           max_refine=8):
        """Batched form on host arrays (pinned arrays copy fastest); returns u."""
        qm = self.mesh.qm
        f = np.ascontiguousarray(forcing, dtype=np.float64)
        nz = f.shape[0]
        u = out if out is not None else np.zeros_like(f)  # the Nyquist plane is left as passed
        b = self._bc_array(bc, nz)
        st = SolveStats()
        rc = lib.sx_field_solve_batched_host(self.h, _dptr(u), _dptr(f),
                                             _dptr(b) if b is not None else None, nz, qm.nplane,
                                             precision, tol_rel, max_refine, C.byref(st))
        _check(rc, "sx_field_solve_batched_host", allow=(OK, WARN_STEP_LIMIT))
        self.last_stats = st.as_dict()
        return u

    def tune(self, inner_iters=None, band_cluster=None, mixed_route=None, band_stages=None, band_lead=None,
             host_chunk=None):
        """Schedule knobs of the batched forms (None leaves a knob alone, 0
        restores its default).  mixed_route: ROUTE_AUTO (by cost), ROUTE_CG
        (FP32 CG for every mode), ROUTE_BAND (band Cholesky for every
        factored mode).  band_lead: K >= 2, the cluster leader taking the last
        of every K band tiles off the critical path (1: none).  host_chunk:
        modes per chunk of solve_batched_host's copy/solve pipeline."""
        if host_chunk is not None:
            _check(lib.sx_modal_tune(self.h, TUNE_HOST_CHUNK, int(host_chunk)), "sx_modal_tune")
        if band_lead is not None:
            _check(lib.sx_modal_tune(self.h, TUNE_BAND_LEAD, int(band_lead)), "sx_modal_tune")
        if inner_iters is not None:
            _check(lib.sx_modal_tune(self.h, TUNE_INNER_ITERS, int(inner_iters)), "sx_modal_tune")
        if band_cluster is not None:
            _check(lib.sx_modal_tune(self.h, TUNE_BAND_CLUSTER, int(band_cluster)), "sx_modal_tune")
        if mixed_route is not None:
            _check(lib.sx_modal_tune(self.h, TUNE_MIXED_ROUTE, int(mixed_route)), "sx_modal_tune")
        if band_stages is not None:
            _check(lib.sx_modal_tune(self.h, TUNE_BAND_STAGES, int(band_stages)), "sx_modal_tune")

    def autotune(self, d_u, d_f, d_bc, nz, stride, precision=FP64, tol_rel=1e-12, max_refine=20, stream=0):
        """Time the batched form's candidate schedules on this data (device
        pointers; d_f is only read) and keep the fastest; returns the choice."""
        r = TuneResult()
        _check(lib.sx_modal_autotune(self.h, d_u, d_f, d_bc, nz, stride, precision, tol_rel, max_refine,
                                     stream, C.byref(r)), "sx_modal_autotune")
        return r.as_dict()

    def profile_band_sweeps(self, reps, stream=0):
        _check(lib.sx_profile_band_sweeps(self.h, reps, stream), "sx_profile_band_sweeps")

    def profile_mixed_iterations(self, reps, stream=0):
        _check(lib.sx_profile_mixed_iterations(self.h, reps, stream), "sx_profile_mixed_iterations")

    def status(self):
        return _check(lib.sx_modal_status(self.h), "sx_modal_status")

    def close(self):
        if getattr(self, "h", None) and lib is not None:
            lib.sx_modal_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def transform_z(d_data, nz, plane_stride, npts=None, sign=1, stream=0):
    """z-direction transform of nz device planes in place (dDFTr,
    femlib/fourier.c:47-171): sign=+1 physical -> Fourier (1/nz, semtex
    plane order), sign=-1 back."""
    _check(lib.sx_transform_z(d_data, nz, plane_stride, plane_stride if npts is None else npts, sign, stream),
           "sx_transform_z")


def _ptrs(ptrs):
    return (C.c_void_p * len(ptrs))(*[int(x) for x in ptrs])


def field_gradient(mesh, d_data, nz, stride, dir, beta=1.0, base_mode=0, stream=0):
    """AuxField::gradient (src/auxfield.cpp:514-616) in place on nz device
    planes: dir 0 d/dx, 1 d/dy, 2 d/dz of Fourier planes."""
    _check(lib.sx_field_gradient(mesh.h, d_data, nz, stride, dir, beta, base_mode, stream), "sx_field_gradient")


def pressure_forcing(mesh, d_us, d_out, nz, stride, dt, beta=1.0, base_mode=0, stream=0):
    """setPForce (dns/integrate.cpp:262-277): d_out = div(us) / dt, us the
    len(d_us) (2 or 3) velocity components."""
    _check(lib.sx_dns_pressure_forcing(mesh.h, _ptrs(d_us), len(d_us), d_out, nz, stride, dt, beta, base_mode,
                                       stream), "sx_dns_pressure_forcing")


def project(mesh, d_us, d_p, d_uf, nz, stride, dt, kinvis, ndim, ncom=None, prandtl=1.0, beta=1.0,
            base_mode=0, stream=0):
    """project (dns/integrate.cpp:280-310): uf[i] = -us[i]/(dt kinvis)
    (times prandtl for a scalar after the ncom velocities) + grad_i(p)/kinvis
    for i < ndim."""
    ncom = len(d_us) if ncom is None else ncom
    _check(lib.sx_dns_project(mesh.h, _ptrs(d_us), d_p, _ptrs(d_uf), ndim, ncom, len(d_us), nz, stride, dt,
                              kinvis, prandtl, beta, base_mode, stream), "sx_dns_project")


def field_smooth(mesh, d_data, nz, stride, stream=0):
    """Field::smooth (src/field.cpp:190-276) in place on nz device planes."""
    _check(lib.sx_field_smooth(mesh.h, d_data, nz, stride, stream), "sx_field_smooth")


def wave_prop(d_us, d_uf, d_h, npts, dt, stream=0):
    """waveProp (dns/integrate.cpp:227-259): d_us[q][i], d_uf[q][i] = level
    q of field i (order = len(d_us) levels), d_h[i] the results."""
    order, nadv = len(d_us), len(d_h)
    us = [x for lev in d_us for x in lev]
    uf = [x for lev in d_uf for x in lev]
    if len(us) != order * nadv or len(uf) != order * nadv:
        raise ValueError("every level needs one pointer per field")
    _check(lib.sx_dns_wave_prop(_ptrs(us), _ptrs(uf), _ptrs(d_h), nadv, order, npts, dt, stream),
           "sx_dns_wave_prop")


def write_field(path, fields, np_, nel, session="semtex_b200", step=0, time=0.0, dt=0.0, kinvis=0.0,
                beta=0.0):
    """Write a field file in the reference's format (sx_field_write).
    fields: {name (one character): (nz, nel*np*np) array}, in file order."""
    names = "".join(fields)
    arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1, nel * np_ * np_) for a in fields.values()]
    nz = arrs[0].shape[0]
    h = FieldHeader(session.encode()[:255], np_, nz, nel, step, time, dt, kinvis, beta, names.encode(), 0)
    ptrs = (C.POINTER(C.c_double) * len(arrs))(*[_dptr(a) for a in arrs])
    _check(lib.sx_field_write(str(path).encode(), C.byref(h), ptrs, nel * np_ * np_), "sx_field_write")


def read_field(path):
    """Read a field file (sx_field_read): (header dict, {name: (nz, nel*np*np) array})."""
    h = FieldHeader()
    _check(lib.sx_field_read_header(str(path).encode(), C.byref(h)), "sx_field_read_header")
    n = h.nel * h.np * h.np
    arrs = [np.zeros((h.nz, n)) for _ in h.fields.decode()]
    ptrs = (C.POINTER(C.c_double) * len(arrs))(*[_dptr(a) for a in arrs])
    _check(lib.sx_field_read(str(path).encode(), C.byref(h), ptrs, n), "sx_field_read")
    return h.as_dict(), dict(zip(h.fields.decode(), arrs))


def field_norms(mesh, d_computed, d_exact, nz, stride, stream=0):
    """compare-style norms of exact - computed per plane on the GPU
    (sx_field_norms): array (nz, 2) of (inf, L2)."""
    out = np.zeros(2 * nz)
    _check(lib.sx_field_norms(mesh.h, d_computed, d_exact, nz, stride, _dptr(out), stream), "sx_field_norms")
    return out.reshape(nz, 2)


def write_numbering(path, sets, fields=None, optimization=3):
    """Write a numbering file (session.num) in enumerate's layout
    (sx_numbering_write).  sets: {set name (e.g. "uv"): QuadMesh}, meshes of
    one geometry whose btog/bmask/nglobal/nsolve/nband are written."""
    names = list(sets)
    ms = [sets[k] for k in names]
    m0 = ms[0]
    bt = [np.ascontiguousarray(m.btog, dtype=np.int32).reshape(-1) for m in ms]
    bm = [np.ascontiguousarray(m.bmask, dtype=np.int32).reshape(-1) for m in ms]
    n = len(ms)
    cn = (C.c_char_p * n)(*[k.encode() for k in names])
    pb = (C.POINTER(C.c_int) * n)(*[_iptr(a) for a in bt])
    pm = (C.POINTER(C.c_int) * n)(*[_iptr(a) for a in bm])
    ng = (C.c_int * n)(*[m.nglobal for m in ms])
    ns = (C.c_int * n)(*[m.nsolve for m in ms])
    nb = (C.c_int * n)(*[m.nband for m in ms])
    _check(lib.sx_numbering_write(str(path).encode(), (fields or "".join(names)).encode(), n, cn, m0.nel, m0.np,
                                  pb, pm, ng, ns, nb, optimization), "sx_numbering_write")


def read_numbering(path, field, nel, np_):
    """Read the number set of `field` from a numbering file
    (sx_numbering_read): dict of btog, bmask (nel, 4(np-1)), nglobal, nsolve,
    nband and the set's name."""
    nx = 4 * (np_ - 1)
    bt = np.zeros(nel * nx, dtype=np.int32)
    bm = np.zeros(nel * nx, dtype=np.int32)
    ng, ns, nb = C.c_int(), C.c_int(), C.c_int()
    name = C.create_string_buffer(64)
    _check(lib.sx_numbering_read(str(path).encode(), field.encode(), nel, np_, _iptr(bt), _iptr(bm), C.byref(ng),
                                 C.byref(ns), C.byref(nb), name, 64), "sx_numbering_read")
    return {"btog": bt.reshape(nel, nx), "bmask": bm.reshape(nel, nx), "nglobal": ng.value,
            "nsolve": ns.value, "nband": nb.value, "set": name.value.decode()}


def with_numbering(qm: QuadMesh, num):
    """A copy of mesh qm numbered by `num` (read_numbering's result)."""
    import dataclasses
    return dataclasses.replace(qm, btog=num["btog"].astype(np.int32), bmask=num["bmask"].astype(np.int32),
                               nglobal=num["nglobal"], nsolve=num["nsolve"], nband=num["nband"])


class Batch:
    """Multi-mesh batch (sx_batch_solve): the planes of several modal systems
    -- different meshes, element counts, orders and mode sets -- solved
    together, each kernel launched once per element order over all members.
    Holds the tables and captured graphs between calls."""

    def __init__(self):
        h = C.c_void_p()
        _check(lib.sx_batch_create(C.byref(h)), "sx_batch_create")
        self.h = h

    def solve(self, members, precision=MIXED_FP32, tol_rel=1e-12, max_refine=20, stream=0):
        """members: sequence of (modal, d_u, d_f, d_bc, nz, stride) with device
        pointers as ints (d_bc may be None).  Returns one stats dict per member."""
        n = len(members)
        mods = (C.c_void_p * n)(*[m[0].h for m in members])
        du = (C.c_void_p * n)(*[m[1] for m in members])
        df = (C.c_void_p * n)(*[m[2] for m in members])
        bcs = [m[3] for m in members]
        dbc = (C.c_void_p * n)(*[b if b else None for b in bcs]) if any(bcs) else None
        nzs = (C.c_int * n)(*[m[4] for m in members])
        strides = (C.c_int * n)(*[m[5] for m in members])
        st = (SolveStats * n)()
        rc = lib.sx_batch_solve(self.h, n, mods, du, df, dbc, nzs, strides, precision, tol_rel, max_refine,
                                stream, st)
        _check(rc, "sx_batch_solve", allow=(OK, WARN_STEP_LIMIT))
        return [s.as_dict() for s in st]

    def close(self):
        if getattr(self, "h", None) and lib is not None:
            lib.sx_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class Server:
    """Continuous-batching request loop (sx_server_*): requests of any mesh,
    order and mode count are admitted as device slots and memory free up;
    each slot solves up to max_batch of them together as one multi-mesh
    batch; geometry and systems stay resident across requests.
    """

    def __init__(self, slots=8, precision=MIXED_FP32, hbm_budget=0, tol_rel=1e-12,
                 max_refine=30, inner_iters=12, max_batch=8):
        cfg = ServerConfig(int(hbm_budget), slots, precision, tol_rel, max_refine, inner_iters, max_batch)
        h = C.c_void_p()
        _check(lib.sx_server_create(C.byref(cfg), C.byref(h)), "sx_server_create")
        self.h = h
        self._live = {}

    def submit(self, qm: QuadMesh, lambda2_modes, betak2_modes, forcing, bc=None, base_mode=0):
        """Queue one solve; returns its id.  forcing: (nz, nplane)."""
        d, keep = mesh_desc(qm)
        lam = np.ascontiguousarray(lambda2_modes, dtype=np.float64)
        bk2 = np.ascontiguousarray(betak2_modes, dtype=np.float64)
        f = np.ascontiguousarray(forcing, dtype=np.float64).reshape(-1, qm.nplane)
        nz = f.shape[0]
        u = np.zeros_like(f)
        b = None
        if bc is not None:
            nb = max(len(qm.boundaries), 1)
            b = np.ascontiguousarray(np.broadcast_to(bc, (nz, nb, qm.np)), dtype=np.float64)
        req = Request(C.pointer(d), base_mode, len(lam), _dptr(lam), _dptr(bk2), nz, qm.nplane,
                      _dptr(f), _dptr(b) if b is not None else None, _dptr(u))
        rid = C.c_ulonglong()
        _check(lib.sx_server_submit(self.h, C.byref(req), C.byref(rid)), "sx_server_submit")
        self._live[rid.value] = u          # the output buffer must outlive the request
        return rid.value

    def wait(self, rid, timeout_s=-1.0):
        """(status, latency_ms, u) of a submitted request."""
        st, lat = C.c_int(), C.c_double()
        _check(lib.sx_server_wait(self.h, rid, timeout_s, C.byref(st), C.byref(lat)), "sx_server_wait")
        return st.value, lat.value, self._live.pop(rid)

    def stats(self):
        s = ServerStats()
        _check(lib.sx_server_get_stats(self.h, C.byref(s)), "sx_server_get_stats")
        return s.as_dict()

    def close(self):
        if getattr(self, "h", None) and lib is not None:
            lib.sx_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
