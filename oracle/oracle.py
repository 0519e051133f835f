"""ctypes front-end to the CPU oracle (oracle/sx_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, as the checker.  The product never
imports this module.

The plane loop below restates ``Field::solve`` (src/field.cpp:557-724) over a
``ModalMatrixSys`` (src/matrix.cpp:33-110): plane 1 (Nyquist) is skipped,
planes 2k and 2k+1 (Re, Im of mode k) share one system with
betak2 = (beta k)^2 (src/field.cpp:1121-1139).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    so = os.path.join(_HERE, "libsx_oracle.so")
    src = os.path.join(_HERE, "sx_oracle.c")
    if force or not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "libsx_oracle.so"])
    return so


def lib():
    global _LIB
    if _LIB is None:
        so = build()
        L = C.CDLL(so)
        L.orc_gll.argtypes = [C.c_int, _dp, _dp, _dp]
        L.orc_gll.restype = C.c_int
        L.orc_mesh_create.argtypes = [C.c_int, C.c_int, _dp, _dp, _ip, _ip, C.c_int, C.c_int, C.c_int,
                                      C.c_int, _ip, _ip, _ip, _dp, _dp, C.POINTER(C.c_int)]
        L.orc_mesh_create.restype = C.c_void_p
        L.orc_mesh_destroy.argtypes = [C.c_void_p]
        L.orc_mesh_geom.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.orc_mesh_geom.restype = C.c_int
        L.orc_boundary_area.argtypes = [C.c_void_p, _dp]
        L.orc_element_matrix.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp]
        L.orc_helmholtz_op.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, _dp, _dp]
        L.orc_sys_create.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.POINTER(C.c_int)]
        L.orc_sys_create.restype = C.c_void_p
        L.orc_sys_destroy.argtypes = [C.c_void_p]
        L.orc_sys_nsolve.argtypes = [C.c_void_p]
        L.orc_sys_nsolve.restype = C.c_int
        L.orc_sys_singular.argtypes = [C.c_void_p]
        L.orc_sys_singular.restype = C.c_int
        L.orc_sys_band.argtypes = [C.c_void_p, _dp]
        L.orc_sys_set_band.argtypes = [C.c_void_p, _dp]
        L.orc_sys_hbi.argtypes = [C.c_void_p, _dp]
        L.orc_sys_hii.argtypes = [C.c_void_p, _dp]
        L.orc_sys_pc.argtypes = [C.c_void_p, _dp]
        L.orc_solve_plane.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_double, C.c_int]
        L.orc_solve_plane.restype = C.c_int
        L.orc_global_op.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_dpbtrf.argtypes = [C.c_int, C.c_int, _dp, C.c_int]
        L.orc_dpbtrf.restype = C.c_int
        L.orc_dpbtrs.argtypes = [C.c_int, C.c_int, _dp, C.c_int, _dp]
        _LIB = L
    return _LIB


def gll(np_: int):
    z = np.zeros(np_)
    w = np.zeros(np_)
    D = np.zeros(np_ * np_)
    lib().orc_gll(np_, z, w, D)
    return z, w, D.reshape(np_, np_)


DIRECT, JACPCG = 0, 1


class OracleMesh:
    """Elements + NumberSys + boundaries, from a semtex_b200.mesh.QuadMesh."""

    def __init__(self, m):
        self.m = m
        nb, be, bs, bk, bK, bC = m.bc_arrays()
        info = C.c_int(0)
        self._keep = [np.ascontiguousarray(a) for a in (m.x.reshape(-1), m.y.reshape(-1),
                                                          m.btog.reshape(-1), m.bmask.reshape(-1))]
        self.h = lib().orc_mesh_create(m.np, m.nel, self._keep[0], self._keep[1],
                                       self._keep[2].astype(np.int32), self._keep[3].astype(np.int32),
                                       m.nglobal, m.nsolve, m.nband, nb, be, bs, bk, bK, bC,
                                       C.byref(info))
        if info.value:
            raise RuntimeError(f"oracle mesh setup failed ({info.value})")

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_mesh_destroy(self.h)
            self.h = None

    def geom(self, e):
        n = self.m.npnp
        arrs = [np.zeros(n) for _ in range(5)]
        has_q3 = lib().orc_mesh_geom(self.h, e, *arrs)
        return arrs, has_q3

    def boundary_area(self):
        a = np.zeros(max(len(self.m.boundaries), 1) * self.m.np)
        lib().orc_boundary_area(self.h, a)
        return a.reshape(-1, self.m.np)


class OracleSystem:
    """One MatrixSys (src/matrix.cpp:139-317) for (lambda2, betak2).

    factor="restated" factors the band with the oracle's own dpbtf2
    restatement; factor="lapack" assembles the same band and factors it with
    LAPACK's dpbtrf from scipy's bundled OpenBLAS -- the routine the reference
    calls (src/matrix.cpp:259) -- which is blocked and far faster on large
    bands (the factor is set-up; solves use the oracle's dpbtrs restatement
    either way)."""

    def __init__(self, mesh: OracleMesh, lambda2: float, betak2: float, method: int = DIRECT,
                 factor: str = "restated"):
        self.mesh = mesh
        self.lambda2, self.betak2, self.method = lambda2, betak2, method
        info = C.c_int(0)
        lapack = method == DIRECT and factor == "lapack"
        self.h = lib().orc_sys_create(mesh.h, lambda2, betak2, 2 if lapack else method, C.byref(info))
        if info.value:
            lib().orc_sys_destroy(self.h)
            self.h = None
            raise RuntimeError(f"oracle system setup failed (info={info.value})")
        self.nsolve = lib().orc_sys_nsolve(self.h)
        self.singular = bool(lib().orc_sys_singular(self.h))
        if lapack and self.nsolve:
            from scipy.linalg.lapack import dpbtrf
            H = self.band()                      # (nsolve, nband) row-major = LAPACK (ldab, n)
            c, info2 = dpbtrf(H.T, lower=0, overwrite_ab=1)
            if info2:
                raise RuntimeError(f"oracle system setup failed (dpbtrf info={info2})")
            lib().orc_sys_set_band(self.h, np.ascontiguousarray(c.T))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_sys_destroy(self.h)
            self.h = None

    def band(self):
        H = np.zeros(self.nsolve * self.mesh.m.nband)
        lib().orc_sys_band(self.h, H)
        return H.reshape(self.nsolve, self.mesh.m.nband)

    def solve_plane(self, forcing, bc, unknown=None, tol_rel=1e-8, step_max=500):
        m = self.mesh.m
        f = np.ascontiguousarray(forcing, dtype=np.float64).reshape(-1).copy()
        u = (np.zeros(m.nplane) if unknown is None
             else np.ascontiguousarray(unknown, dtype=np.float64).reshape(-1).copy())
        nb = max(len(m.boundaries), 1)
        if bc is None:
            b = np.zeros(nb * m.np)
        else:
            b = np.ascontiguousarray(bc, dtype=np.float64).reshape(-1)
        if b.size != nb * m.np:
            raise ValueError(f"bc has {b.size} values, expected nbound*np = {nb * m.np}")
        it = lib().orc_solve_plane(self.h, u, f, b, tol_rel, step_max)
        return u, it


def mode_constant(beta: float, mode: int) -> float:
    """betak2 = (beta k)^2 for Cartesian geometry (src/field.cpp:1121-1139)."""
    return (beta * mode) ** 2


def solve_planes(mesh: OracleMesh, lambda2, beta, forcing, bc, method=DIRECT,
                 tol_rel=1e-8, step_max=500, lambda2_per_mode=None, unknown=None):
    """Field::solve over nz planes in semtex Fourier order.

    forcing : (nz, nplane); bc : (nz, nbound, np) or None.  Plane 1 (Nyquist)
    is left zero.  ``lambda2_per_mode`` overrides lambda2 mode by mode (one
    MatrixSys per mode, betak2 still (beta k)^2).
    Returns (u (nz, nplane), iterations per plane).
    """
    m = mesh.m
    forcing = np.asarray(forcing, dtype=np.float64).reshape(-1, m.nplane)
    nz = forcing.shape[0]
    out = np.zeros_like(forcing)
    iters = np.zeros(nz, dtype=np.int64)
    nb = max(len(m.boundaries), 1)
    if bc is None:
        bc = np.zeros((nz, nb, m.np))
    systems = {}
    for k in range(nz):
        if k == 1:
            continue
        mode = k >> 1
        lam = lambda2 if lambda2_per_mode is None else lambda2_per_mode[mode]
        if mode not in systems:
            systems[mode] = OracleSystem(mesh, lam, mode_constant(beta, mode), method)
        u0 = None if unknown is None else unknown[k]
        out[k], iters[k] = systems[mode].solve_plane(forcing[k], bc[k], u0, tol_rel, step_max)
    return out, iters


def transform_z(data, sign):
    """dDFTr (femlib/fourier.c:47-171) restated as a direct DFT along axis 0
    of `data` (nz planes x points), the checker for sx_transform_z.

    Forward (sign=+1): X_k = (1/nz) sum_j x_j exp(-2 pi i j k / nz) -- the
    sign of DMPFFT's DGPFA call (femlib/temfftd.F:218-238) -- stored as
    plane 0 = Re X_0, plane 1 = Re X_{nz/2}, planes 2k, 2k+1 = Re X_k,
    Im X_k (fourier.c:58-63).  Inverse (sign=-1): the unscaled sum back.
    """
    x = np.asarray(data, dtype=np.float64)
    nz = x.shape[0]
    if nz == 1:
        return x.copy()
    assert nz % 2 == 0
    nh = nz // 2
    j = np.arange(nz)
    out = np.empty_like(x)
    if sign == 1:
        for k in range(nh + 1):
            ang = 2.0 * np.pi * ((j * k) % nz) / nz
            re = (np.cos(ang) @ x) / nz
            im = (-np.sin(ang) @ x) / nz
            if k == 0:
                out[0] = re
            elif k == nh:
                out[1] = re
            else:
                out[2 * k] = re
                out[2 * k + 1] = im
        return out
    out[:] = x[0] + np.where(j % 2 == 0, 1.0, -1.0)[:, None] * x[1]
    for k in range(1, nh):
        ang = 2.0 * np.pi * ((j * k) % nz) / nz
        out += 2.0 * (np.cos(ang)[:, None] * x[2 * k] - np.sin(ang)[:, None] * x[2 * k + 1])
    return out
